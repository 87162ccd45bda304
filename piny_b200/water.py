"""Flexible point-charge water boxes: models, seeded synthetic configurations
and PINY input directories.

Units follow PINY: inputs in Angstrom / Kelvin (energies divided by k_B),
internal arrays in Bohr / Hartree (``BOHR``, ``BOLTZ`` as defined in PINY's
include/typ_defs/defines.h:76-79).

The PINY input writer mirrors python/piny/tools.py:137-182 (``input_str``,
``write_input_directory``, ``initial_file``) so that PINY itself can be run on
exactly the configuration the device path sees.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

BOHR = 0.529177          # Angstrom per Bohr (defines.h:76)
BOLTZ = 315777.0         # Kelvin per Hartree (defines.h:78)
KB_KCAL = 0.001987204118  # kcal/mol/K (examples/q-TIP4P-F/water-q-TIP4P-F.py:1)
AMU = 1.66053906660e-27
HBAR = 1.054571817e-34
KB_SI = 1.380649e-23


@dataclass
class WaterModel:
    name: str
    sites: list            # site names in molecule order
    masses: list
    charges: list
    lj_sigma: float        # Angstrom (O-O only)
    lj_eps_kcal: float     # kcal/mol
    bond: dict             # {"type": "harm", "r0", "k"} or {"type": "quartic", "r0", "D", "a"}
    bend_theta0: float     # degrees
    bend_k_kcal: float     # kcal/mol/rad^2, V = k/2 (theta-theta0)^2
    ghost: dict = field(default_factory=dict)  # site index -> [(comp index, coef)]

    @property
    def nsite(self):
        return len(self.sites)

    @property
    def type_names(self):
        seen = []
        for s in self.sites:
            if s not in seen:
                seen.append(s)
        return seen


SPC_FW = WaterModel(
    name="q-SPC/Fw", sites=["O", "H", "H"], masses=[15.999, 1.008, 1.008],
    charges=[-0.84, 0.42, 0.42], lj_sigma=3.1655, lj_eps_kcal=0.1554,
    bond={"type": "harm", "r0": 1.0, "k": 1059.162},
    bend_theta0=112.0, bend_k_kcal=75.9)

TIP4P_F = WaterModel(
    name="q-TIP4P/F", sites=["O", "H", "H", "M"], masses=[15.999, 1.008, 1.008, 1.0],
    charges=[0.0, 0.5564, 0.5564, -1.1128], lj_sigma=3.1589, lj_eps_kcal=0.1852,
    bond={"type": "quartic", "r0": 0.9419, "D": 116.09, "a": 2.287},
    bend_theta0=107.4, bend_k_kcal=87.85,
    ghost={3: [(0, 0.73612), (1, 0.13194), (2, 0.13194)]})

MODELS = {"spcfw": SPC_FW, "tip4pf": TIP4P_F}


@dataclass
class BoxSpec:
    """One periodic box of flexible water and its PINY settings."""
    model: WaterModel
    nmol: int
    L: float                 # cubic box edge, Angstrom
    nbeads: int = 1
    temperature: float = 300.0
    seed: int = 12345
    cutoff: float = 9.0      # Angstrom (max_dist of every .inter pair)
    min_dist: float = 0.1    # Angstrom (inner end of the spline tables)
    skin: float = 1.0        # Angstrom (verlist_skin)
    alpha: float = 0.35      # 1/Angstrom
    grid: int = 32           # PME grid points per edge
    order: int = 6           # PME interpolation order
    kmax: int = 0            # ewald_kmax (0: grid/2 - 2)
    nsplin: int = 2000       # inter_spline_pts (PINY default)
    jitter: float = 0.05     # Angstrom
    update_type: str = "lnk_list"
    kmax_pme_in: int = 0     # ewald_kmax_pme override (0: derived from ``grid``)

    @property
    def natm(self):
        return self.nmol * self.model.nsite

    @property
    def kmax_ewald(self):
        return self.kmax if self.kmax > 0 else self.grid // 2 - 2

    @property
    def kmax_pme(self):
        if self.kmax_pme_in > 0:
            return self.kmax_pme_in
        # set_pme_grid (set_cp_ewald.c:204-300) gives 4*(NINT(kmax_pme/2)+1)
        # points for a cubic box; 2*(grid/4 - 1) reproduces ``grid``.
        return 2 * (self.grid // 4 - 1)


# ---------------------------------------------------------------------------
# configurations

def _random_rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def molecule_template(model: WaterModel):
    """Equilibrium geometry (Angstrom), O at the origin, HOH in the xy plane."""
    r0 = model.bond["r0"]
    th = math.radians(model.bend_theta0)
    O = np.zeros(3)
    H1 = r0 * np.array([math.sin(th / 2), math.cos(th / 2), 0.0])
    H2 = r0 * np.array([-math.sin(th / 2), math.cos(th / 2), 0.0])
    sites = [O, H1, H2]
    if model.nsite == 4:
        sites.append(np.zeros(3))
    return np.array(sites)


def apply_ghosts(model: WaterModel, pos):
    """M site = sum_k c_k r_k (PINY get_ghost_pos, ghost_control.c:28-69)."""
    if not model.ghost:
        return pos
    ns = model.nsite
    p = pos.reshape(pos.shape[:-2] + (-1, ns, 3))
    for g, comps in model.ghost.items():
        acc = np.zeros_like(p[..., g, :])
        for c, coef in comps:
            acc = acc + coef * p[..., c, :]
        p[..., g, :] = acc
    return p.reshape(pos.shape)


def ring_polymer_displacements(rng, masses_amu, nbeads, temperature):
    """Free ring-polymer bead displacements (Angstrom), shape (P, N, 3).

    Mode j of P has variance hbar^2 beta / (m P 4 sin^2(pi j/P)); the centroid
    mode is zero so every atom's beads are centred on its classical position.
    """
    P = nbeads
    N = len(masses_amu)
    if P == 1:
        return np.zeros((1, N, 3))
    beta = 1.0 / (KB_SI * temperature)
    m = np.asarray(masses_amu) * AMU
    # orthonormal real normal-mode basis C[k, j]
    k = np.arange(P)
    C = np.zeros((P, P))
    C[:, 0] = 1.0 / math.sqrt(P)
    col = 1
    freq = [0.0]
    for j in range(1, (P - 1) // 2 + 1):
        C[:, col] = math.sqrt(2.0 / P) * np.cos(2 * math.pi * j * k / P)
        C[:, col + 1] = math.sqrt(2.0 / P) * np.sin(2 * math.pi * j * k / P)
        freq += [j, j]
        col += 2
    if P % 2 == 0:
        C[:, col] = np.cos(math.pi * k) / math.sqrt(P)
        freq.append(P // 2)
    freq = np.array(freq, dtype=float)
    var = np.zeros(P)
    var[1:] = 1.0 / (4.0 * np.sin(math.pi * freq[1:] / P) ** 2)
    # per-atom scale hbar^2 beta / (m P), in Angstrom^2
    scale = (HBAR ** 2 * beta / (m * P)) * 1e20
    q = rng.normal(size=(P, N, 3)) * np.sqrt(var)[:, None, None] * np.sqrt(scale)[None, :, None]
    return np.einsum("kj,jna->kna", C, q)


def build_positions(spec: BoxSpec):
    """Seeded synthetic configuration, Angstrom, shape (P, natm, 3)."""
    rng = np.random.default_rng(spec.seed)
    model = spec.model
    n = spec.nmol
    m = int(math.ceil(round(n ** (1.0 / 3.0), 9)))
    while m ** 3 < n:
        m += 1
    a = spec.L / m
    idx = np.arange(n)
    lattice = np.stack([idx % m, (idx // m) % m, idx // (m * m)], axis=1) * a + 0.5 * a
    tmpl = molecule_template(model)
    com = (tmpl[:3] * np.array(model.masses[:3])[:, None]).sum(0) / sum(model.masses[:3])
    tmpl = tmpl - com
    R = _random_rotations(rng, n)
    mol = np.einsum("nij,sj->nsi", R, tmpl) + lattice[:, None, :]
    mol = mol + rng.normal(scale=spec.jitter, size=mol.shape)
    pos = mol.reshape(n * model.nsite, 3)
    masses = np.tile(model.masses, n)
    beads = pos[None] + ring_polymer_displacements(rng, masses, spec.nbeads, spec.temperature)
    beads = apply_ghosts(model, beads)
    return beads


# ---------------------------------------------------------------------------
# PINY input directory (python/piny/tools.py:137-182 formats)

def _input_str(sections):
    out = []
    for name, sec in sections:
        lines = ["    \\%s{%s}" % (k, v) for k, v in sec.items()]
        out.append("~%s[\n" % name + "\n".join(lines) + "]")
    return "\n\n".join(out) + "\n"


def _fmt(x):
    return repr(float(x))


def piny_input_files(spec: BoxSpec, pos_angstrom, sim_typ=None, respa=None):
    """Return {filename: text} for a PINY run of ``spec`` at ``pos_angstrom``.

    ``respa`` (optional) switches on PINY's RESPA split: a dict with the step
    counts ``lrf``, ``intra``, ``pimd`` (respa_steps_lrf / _intra / _pimd),
    ``rheal`` (respa_rheal, Angstrom) and ``eq_res`` (the bond's eq_res
    shift, Angstrom), and optionally ``kmax_res`` (ewald_respa_kmax, the
    reciprocal-space RESPA set) with ``pme_res`` = (ewald_respa_kmax_pme,
    ewald_respa_interp_pme) for PINY's separate RESPA PME grid; the inner
    cutoff is each pair's ``res_dist``."""
    model = spec.model
    P = spec.nbeads
    L = spec.L
    if sim_typ is None:
        sim_typ = "pimd" if P > 1 else "md"
    gen = {
        "simulation_typ": sim_typ, "ensemble_typ": "nvt", "num_time_step": 1,
        "restart_type": "initial", "time_step": 0.5, "temperature": spec.temperature,
        "generic_fft_opt": "on", "num_proc_tot": 1, "num_proc_beads": 1,
        "num_proc_class_forc": 1,
    }
    sections = [("sim_gen_def", gen)]
    if P > 1:
        sections.append(("sim_pimd_def", {
            "path_int_beads": P, "path_int_md_typ": "centroid",
            "initial_spread_opt": "off", "respa_steps_pimd": int(respa["pimd"]) if respa else 1}))
    if respa:
        sections.append(("sim_run_def", {
            "respa_steps_lrf": int(respa["lrf"]), "respa_steps_torsion": 1,
            "respa_steps_intra": int(respa["intra"]), "respa_rheal": _fmt(respa["rheal"])}))
    sections += [
        ("sim_list_def", {"neighbor_list": "ver_list", "verlist_skin": _fmt(spec.skin),
                          "update_type": spec.update_type}),
        ("sim_vol_def", {"periodicity": 3}),
        ("sim_class_PE_def", {
            "shift_inter_pe": "swit", "inter_spline_pts": spec.nsplin,
            "ewald_alpha": _fmt(spec.alpha * L), "ewald_kmax": spec.kmax_ewald,
            "ewald_pme_opt": "on", "ewald_kmax_pme": spec.kmax_pme,
            "ewald_interp_pme": spec.order, "ewald_respa_pme_opt": "off",
            "inter_PE_calc_freq": 1, "sep_VanderWaals": "on",
            **({"ewald_respa_kmax": int(respa["kmax_res"])} if respa and respa.get("kmax_res") else {}),
            **({"ewald_respa_pme_opt": "on", "ewald_respa_kmax_pme": int(respa["pme_res"][0]),
                "ewald_respa_interp_pme": int(respa["pme_res"][1])} if respa and respa.get("pme_res") else {})}),
        ("sim_nhc_def", {"atm_nhc_tau_def": 20.0, "atm_nhc_len": 4, "respa_steps_nhc": 1,
                         "yosh_steps_nhc": 3, "respa_xi_opt": 1}),
        ("sim_write_def", {
            "sim_name": "water.out", "write_screen_freq": 1000000, "instant_file": "water.iavg",
            "write_inst_freq": 1000000, "atm_pos_file": "water.confp",
            "write_pos_freq": 1000000, "path_cent_file": "water-centroid.confp",
            "path_cent_freq": 1000000, "atm_vel_file": "water.confv",
            "write_vel_freq": 1000000, "atm_force_file": "water.conff",
            "write_force_freq": 1000000, "out_restart_file": "water.restart",
            "write_dump_freq": 1000000, "in_restart_file": "water.initial",
            "mol_set_file": "water.set", "conf_file_format": "formatted"}),
    ]
    files = {"water.input": _input_str(sections)}

    parm = [("molecule_name_def", {"molecule_name": "water", "natom": model.nsite})]
    for i, s in enumerate(model.sites):
        d = {"atom_typ": s, "atom_ind": i + 1, "mass": model.masses[i], "charge": _fmt(model.charges[i])}
        if i in model.ghost:
            for c, (comp, coef) in enumerate(model.ghost[i]):
                d["def_ghost%d" % (c + 1)] = "%d, %s" % (comp + 1, _fmt(coef))
        parm.append(("atom_def", d))
    parm.append(("bond_def", {"atom1": 1, "atom2": 2}))
    parm.append(("bond_def", {"atom1": 1, "atom2": 3}))
    parm.append(("bend_def", {"atom1": 2, "atom2": 1, "atom3": 3}))
    files["water.parm"] = _input_str(parm)

    b = model.bond
    if b["type"] == "harm":
        bond = {"atom1": "O", "atom2": "H", "pot_type": "harm",
                "fk": _fmt(b["k"] / KB_KCAL), "eq": _fmt(b["r0"])}
    else:
        D = b["D"] / KB_KCAL
        a = b["a"]
        bond = {"atom1": "O", "atom2": "H", "pot_type": "power", "eq": _fmt(b["r0"]),
                "p2": _fmt(D * a ** 2), "p3": _fmt(-D * a ** 3), "p4": _fmt(7.0 * D * a ** 4 / 12.0)}
    if respa:
        bond["eq_res"] = _fmt(respa["eq_res"])
    files["water.bond"] = _input_str([("bond_parm", bond)])
    files["water.bend"] = _input_str([("bend_parm", {
        "atom1": "H", "atom2": "O", "atom3": "H", "pot_type_bend": "harm",
        "fk_bend": _fmt(model.bend_k_kcal / KB_KCAL), "eq_bend": _fmt(model.bend_theta0)})])

    types = model.type_names
    inter = []
    for i, t1 in enumerate(types):
        for t2 in types[i:]:
            d = {"atom1": t1, "atom2": t2, "min_dist": _fmt(spec.min_dist),
                 "max_dist": _fmt(spec.cutoff), "res_dist": _fmt(min(5.0, spec.cutoff - 1.0))}
            if t1 == "O" and t2 == "O":
                d.update({"pot_type": "lennard-jones", "eps": _fmt(model.lj_eps_kcal / KB_KCAL),
                          "sig": _fmt(model.lj_sigma)})
            else:
                d["pot_type"] = "null"
            inter.append(("inter_parm", d))
    files["water.inter"] = _input_str(inter)
    files["water.set"] = _input_str([
        ("molecule_def", {"mol_parm_file": "water.parm", "mol_opt_nhc": "global",
                          "num_mol": spec.nmol, "mol_index": 1, "mol_name": "water"}),
        ("data_base_def", {"bond_file": "water.bond", "bend_file": "water.bend",
                           "inter_file": "water.inter"})])

    natm = spec.natm
    lines = ["%d 1 %d" % (natm, P)]
    for p in range(P):
        for i in range(natm):
            lines.append("%s %s %s" % tuple(_fmt(v) for v in pos_angstrom[p, i]))
    for i in range(3):
        row = [0.0, 0.0, 0.0]
        row[i] = L
        lines.append("%s %s %s" % tuple(_fmt(v) for v in row))
    files["water.initial"] = "\n".join(lines) + "\n"
    return files


def write_piny_input(directory, spec: BoxSpec, pos_angstrom, sim_typ=None, respa=None):
    os.makedirs(directory, exist_ok=True)
    for name, text in piny_input_files(spec, pos_angstrom, sim_typ, respa).items():
        with open(os.path.join(directory, name), "w") as f:
            f.write(text)
    return os.path.join(directory, "water.input")


# ---------------------------------------------------------------------------
# the benchmark configurations (seeded synthetic stand-ins)

def density_box_edge(nmol, density_per_A3=0.03342):
    return (nmol / density_per_A3) ** (1.0 / 3.0)


def c4_specs(nbox: int = 64, seed: int = 2024, nmin: int = 64, nmax: int = 2048):
    """The batched configuration: `nbox` independent q-TIP4P/F boxes with
    molecule counts drawn log-uniformly from [nmin, nmax] and bead counts from
    {1, 4, 8, 16, 32, 64} (seeded), each at 0.997 g/cm^3 (L = (n/0.03342)^(1/3)
    Angstrom) with a PME mesh of the next power of two >= 1 point per
    Angstrom, order 8, and the shared cutoff / skin / alpha.  Box i uses seed
    seed + i for its geometry."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nbox):
        n = int(round(float(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))))
        P = int(rng.choice([1, 4, 8, 16, 32, 64]))
        L = density_box_edge(n)
        grid = 1 << int(np.ceil(np.log2(L)))
        out.append(BoxSpec(TIP4P_F, n, L, P, 298.0, seed + i, grid=grid, order=8))
    return out


def named_spec(name: str) -> BoxSpec:
    if name == "spcfw_256_p1":
        return BoxSpec(SPC_FW, 256, 19.73, 1, 300.0, 12345, grid=32, order=6)
    if name == "spcfw_256_p32":
        return BoxSpec(SPC_FW, 256, 19.73, 32, 300.0, 12345, grid=32, order=6)
    if name == "tip4pf_4096_p32":
        return BoxSpec(TIP4P_F, 4096, 49.66, 32, 298.0, 12345, grid=64, order=8)
    if name == "tip4pf_1024_p16":
        return BoxSpec(TIP4P_F, 1024, 31.28, 16, 298.0, 12345, grid=32, order=8)
    if name == "tip4pf_1024_p32":
        return BoxSpec(TIP4P_F, 1024, 31.28, 32, 298.0, 12345, grid=32, order=8)
    if name == "tip4pf_256_p4":
        return BoxSpec(TIP4P_F, 256, 19.73, 4, 298.0, 777, grid=32, order=8)
    if name == "spcfw_216_p4":
        return BoxSpec(SPC_FW, 216, 18.64, 4, 300.0, 4242, grid=32, order=6)
    raise KeyError(name)
