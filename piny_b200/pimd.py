"""Set-up data of PINY's NVT ring-polymer step (host side).

The device step (pinyb200_pimd_*, driven by ``lib.DevicePimd``) takes the
products of PINY's set-up stage; this module forms them for a box the way
PINY does:

* ``path_integral_setup``: bead masses, kinetic prefactors and path
  eigenvalues of path_integral_init (src/energy/pimd/transform_cnt.c:23-233);
* ``massive_chains``: chain sets with one Nose-Hoover chain per atom
  coordinate, ghosts on the null chain -- PINY's bead thermostats
  (src/interface/coords/set_atm_NHC.c:648-724) and its class thermostat
  option 6 (set_atm_NHC.c:450-476, expanded and scaled as :506-547);
* ``yoshida_weights``: the stage weights of set_yosh
  (src/integrate/md/int_utils.c:244-302) for 1, 3 and 5 stages, which are
  Suzuki's symmetric compositions w = 1/(2 - 2^(1/3)) and 1/(4 - 4^(1/3)).
  For 7 and 9 stages pass PINY's own ``therm_info.wdti``.

Units are PINY's (atomic units; temperatures in Kelvin, BOLTZ Kelvin per
Hartree).
"""
from __future__ import annotations

import numpy as np

from .lib import NORMAL_MODES, STAGING
from .water import BOLTZ


def path_integral_setup(mass, nbeads: int, kind: int, temperature: float, gamma_adb: float = 1.0, ghost=None):
    """bead_mass [P][natm], prekf [natm], path_eig [P] as path_integral_init
    sets them (the eigenvalue of the centroid is 0 on return, as there)."""
    mass = np.asarray(mass, np.float64)
    P = int(nbeads)
    beta = BOLTZ / temperature
    tau = BOLTZ / (temperature * float(P))
    prekf = mass / (2.0 * tau * beta)
    if ghost is not None:
        prekf = np.where(np.asarray(ghost, bool), 0.0, prekf)
    veig = np.zeros(P + 1)  # 1-based as in PINY
    if kind == NORMAL_MODES:
        tpip = 2.0 * np.pi / float(P)
        pre = 4.0 * float(P)
        veig[1] = 1.0
        if P > 1:
            veig[P] = pre
        for ip in range(2, P // 2 + 1):
            temp = (1.0 - np.cos(tpip * float(ip - 1))) * pre
            veig[2 * ip - 2] = temp
            veig[2 * ip - 1] = temp
    elif kind == STAGING:
        veig[1] = 1.0
        for ip in range(2, P + 1):
            veig[ip] = float(ip) / float(ip - 1)
    else:
        raise ValueError("kind must be STAGING or NORMAL_MODES")
    bead_mass = np.empty((P, len(mass)))
    for ip in range(1, P + 1):
        bead_mass[ip - 1] = mass * veig[ip] if ip == 1 else mass * veig[ip] * gamma_adb * gamma_adb
    veig[1] = 0.0
    return {"bead_mass": bead_mass, "prekf": prekf, "path_eig": veig[1:].copy()}


def yoshida_weights(nyosh: int, dti: float):
    """Stage weights x dti of PINY's set_yosh for 1, 3 or 5 stages."""
    if nyosh == 1:
        w = [1.0]
    elif nyosh == 3:
        t = 2.0 ** (1.0 / 3.0)
        w = [1.0 / (2.0 - t), -t / (2.0 - t), 1.0 / (2.0 - t)]
    elif nyosh == 5:
        p2 = 1.0 / (4.0 - 4.0 ** (1.0 / 3.0))
        w = [p2, p2, 1.0 - 4.0 * p2, p2, p2]
    else:
        raise ValueError("1, 3 or 5 stages here; for 7 or 9 pass PINY's therm_info.wdti")
    return np.array(w) * dti


def massive_chains(natm: int, ghost, temperature: float, first_mass: float, len_nhc: int, nres_nhc: int,
                   wdti, bead_set: bool):
    """One chain per coordinate of every non-ghost atom.  first_mass is
    PINY's unscaled first-link mass: tau^2 T for the class set (option 6),
    BOLTZ^2 gamma^2 / (P T^2) for the bead set."""
    ghost = np.zeros(natm, bool) if ghost is None else np.asarray(ghost, bool)
    real = np.flatnonzero(~ghost)
    num = 3 * len(real)
    inhc = np.full((3, natm), num, np.int32)
    for d in range(3):
        inhc[d, real] = 3 * np.arange(len(real)) + d
    T = float(temperature)
    mass_nhc = np.empty((len_nhc, num))
    gkt = np.empty((len_nhc, num))
    # expansion to len_nhc, then the first link (set_atm_NHC.c:506-547, :713-724)
    mass_nhc[1:] = first_mass * T / BOLTZ if bead_set else first_mass / BOLTZ
    gkt[1:] = T / BOLTZ
    mass_nhc[0] = first_mass * T / BOLTZ if bead_set else first_mass * 1.0 / BOLTZ
    gkt[0] = T / BOLTZ
    return {"num_nhc": num, "len_nhc": len_nhc, "nres_nhc": nres_nhc, "wdti": np.asarray(wdti, np.float64),
            "inhc": inhc, "mass_nhc": mass_nhc, "gkt": gkt}


def nhc_time_step(dt: float, nres=(1, 1, 1, 1), ix_respa: int = 1) -> float:
    """dt_nhc of the chains for RESPA level ix_respa (int_NVT_pimd.c:96-122):
    dt divided by the step counts of the levels down to ix_respa."""
    nt, no, na, np_ = (int(v) for v in nres)
    div = [1, nt, nt * no, nt * no * na, nt * no * na * np_][int(ix_respa) - 1]
    return dt / float(div)


def nvt_setup(mass, ghost, nbeads: int, kind: int, temperature: float, dt: float, tau_nhc: float,
              len_nhc: int = 4, nres_nhc: int = 1, nyosh: int = 3, gamma_adb: float = 1.0,
              nres=(1, 1, 1, 1), ix_respa: int = 1):
    """Everything pinyb200_pimd_create takes for one box: the class set
    thermostats bead 1 per coordinate (PINY option 6), the bead set beads
    2..P (PINY's bead thermostats).  nres = (nres_ter, nres_tor, nres_tra,
    nres_pimd) and ix_respa set PINY's RESPA loops; dt is the outer step."""
    mass = np.asarray(mass, np.float64)
    natm = len(mass)
    ghost = np.zeros(natm, bool) if ghost is None else np.asarray(ghost, bool)
    pis = path_integral_setup(mass, nbeads, kind, temperature, gamma_adb, ghost)
    w = yoshida_weights(nyosh, nhc_time_step(dt, nres, ix_respa) / nres_nhc)
    T = float(temperature)
    cls = massive_chains(natm, ghost, T, tau_nhc * tau_nhc * T, len_nhc, nres_nhc, w, False)
    bead = None
    if nbeads > 1:
        pre = BOLTZ * BOLTZ * gamma_adb * gamma_adb / float(nbeads)
        bead = massive_chains(natm, ghost, T, pre / (T * T), len_nhc, nres_nhc, w, True)
    return {"natm": natm, "nbeads": int(nbeads), "kind": int(kind), "mass": mass, **pis, "wght_pimd": 1.0,
            "dt": float(dt), "beta": BOLTZ / T, "temperature": T, "nfree_atoms": int((~ghost).sum()),
            "class_nhc": cls, "bead_nhc": bead, "nres": tuple(int(v) for v in nres), "ix_respa": int(ix_respa)}
