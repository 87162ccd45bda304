"""ctypes front end of the oracle (liboracle_piny.so).

TEST INFRASTRUCTURE ONLY: the checker for the device path.  Imported by
tests/, the smoke check and the benchmark's CPU-baseline leg, never by the
product package.

A "system" is a dict of numpy arrays/scalars with the field names of
``orc_system`` (piny_oracle.h), 0-based, PINY internal units.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_piny.so")

_i = C.c_int
_d = C.c_double
_pi = C.POINTER(C.c_int)
_pd = C.POINTER(C.c_double)


class OrcSystem(C.Structure):
    _fields_ = [
        ("natm", _i), ("ntyp", _i), ("atm_typ", _pi), ("charge", _pd),
        ("nsplin", _i), ("ninter_unique", _i), ("inter_map", _pi), ("cutoff", _pd),
        ("rmin_spl", _pd), ("dr_spl", _pd), ("dri_spl", _pd),
        ("cv0", _pd), ("cdv0", _pd), ("cv0_c", _pd), ("cdv0_c", _pd),
        ("skin", _d), ("clong", _d), ("iswit_vdw", _i),
        ("excl_off", _pi), ("excl_j", _pi),
        ("alp_ewd", _d), ("self_erf", _d), ("nktot", _i),
        ("kastr", _pi), ("kbstr", _pi), ("kcstr", _pi), ("bweight", _pd),
        ("ngrid_a", _i), ("ngrid_b", _i), ("ngrid_c", _i), ("n_interp", _i),
        ("necor", _i), ("ecor_j1", _pi), ("ecor_j2", _pi), ("ecor_nsplin", _i),
        ("ecor_rmin", _d), ("ecor_dr", _d), ("ecor_dri", _d), ("ecor_cv0", _pd), ("ecor_cdv0", _pd),
        ("nbond", _i), ("bond_j1", _pi), ("bond_j2", _pi), ("bond_typ", _pi), ("nbond_typ", _i),
        ("bond_eq", _pd), ("bond_c", _pd), ("bond_dc", _pd),
        ("nbend", _i), ("bend_j1", _pi), ("bend_j2", _pi), ("bend_j3", _pi), ("bend_typ", _pi),
        ("nbend_typ", _i), ("bend_c", _pd), ("bend_s", _pd), ("bend_dc", _pd), ("bend_ds", _pd),
        ("nghost", _i), ("ghost_ncomp", _i), ("ghost_atom", _pi), ("ghost_comp", _pi), ("ghost_coef", _pd),
    ]


class OrcEnergies(C.Structure):
    _fields_ = [(n, _d) for n in ("vreal", "vvdw", "vcoul", "vrecip", "vself", "vbgr", "vecor",
                                  "vlong", "vbond", "vbend", "vintert", "vintrat")] + [("pvten", _d * 9)]


class OrcRespa(C.Structure):
    _fields_ = [
        ("wght_ter", _d), ("wght_ter_res", _d), ("wght_tra_res", _d),
        ("int_res_ter", _i), ("int_res_inter", _i), ("ires_bond", _i),
        ("cutoff_res", _pd), ("rheal_res", _d), ("bond_eq_res", _pd),
        ("nktot_res", _i), ("ecor_cdv0_res", _pd),
        ("pme_res_on", _i), ("ngrid_res", _i * 3), ("n_interp_res", _i),
        ("kastr_res", _pi), ("kbstr_res", _pi), ("kcstr_res", _pi), ("bweight_res", _pd),
    ]


def build():
    """Compile the oracle restatement (plain gcc)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Oracle:
    def __init__(self):
        if not os.path.exists(LIB):
            build()
        self.lib = C.CDLL(LIB)
        L = self.lib
        L.orc_spline_table.argtypes = [_i, _d, _d, _i, _d, _d, _d, _d, _i, _pd, _pd, _pd, _pd]
        L.orc_ewald_ecut.restype = _d
        L.orc_ewald_ecut.argtypes = [_i, _d]
        L.orc_kmaxv.argtypes = [_d, _pd, _pi]
        L.orc_kvec_count.restype = _i
        L.orc_kvec_count.argtypes = [_d, _pi, _pd]
        L.orc_kvec_fill.restype = _i
        L.orc_kvec_fill.argtypes = [_d, _pi, _pd, _pi, _pi, _pi]
        L.orc_pme_grid.argtypes = [_d, _d, _pd, _pi, _i, _pi]
        L.orc_pme_bweight.argtypes = [_i, _pi, _pi, _pi, _pi, _i, _pd]
        L.orc_pimd_transform.restype = _i
        L.orc_pimd_transform.argtypes = [_i, _i, _i, _i, _pd]
        L.orc_nhc_apply.argtypes = [_i, _pi, _pd, _pd, _i, _i, _i, _i, _pd, _pd, _pd, _pd, _pd]
        L.orc_pimd_springs.restype = _d
        L.orc_pimd_springs.argtypes = [_i, _i, _pd, _pd, _pd, _d, _pd, _pd]
        L.orc_pimd_force_post.restype = _d
        L.orc_pimd_force_post.argtypes = [_i, _i, _i, _pd, _pd, _pd, _pd, _i, _d, _pd, _pd]
        L.orc_pimd_force_post_respa.restype = _d
        L.orc_pimd_force_post_respa.argtypes = [_i, _i, _i, _pd, _pd, _pd, _pd, _pd, _i, _d, _i, _pd, _pd]
        L.orc_ecor_table.argtypes = [_i, _d, _d, _d, _pd, _pd, _pd, _pd, _pd]
        L.orc_gauss_legendre.argtypes = [_i, _pd, _pd]
        L.orc_bond_power.argtypes = [_d, _d, _d, _pd, _pd]
        L.orc_bend_harm.argtypes = [_d, _d, _pd, _pd, _pd, _pd]
        L.orc_clong.restype = _d
        L.orc_clong.argtypes = [_i, _i, _pi, _pd, _pd, _d, _i]
        L.orc_verlist.restype = C.c_long
        L.orc_verlist.argtypes = [C.POINTER(OrcSystem), _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd,
                                  C.c_long, _pi, _pi]
        L.orc_verlist_rows.restype = C.c_long
        L.orc_verlist_rows.argtypes = [C.POINTER(OrcSystem), _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _i, _i,
                                       C.c_long, _pi, _pi]
        L.orc_energy_force.argtypes = [C.POINTER(OrcSystem), _i, _pd, _pd, _pd, C.c_long, _pi, _pi, _i,
                                       _pd, C.POINTER(OrcEnergies)]
        L.orc_respa_force.argtypes = [C.POINTER(OrcSystem), C.POINTER(OrcRespa), _i, _i, _pd, _pd, _pd,
                                      C.c_long, _pi, _pi, _i, _pd, _pd]

    # -- helpers -----------------------------------------------------------
    @staticmethod
    def _d(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        return a, a.ctypes.data_as(_pd)

    @staticmethod
    def _i(a):
        a = np.ascontiguousarray(a, dtype=np.int32)
        return a, a.ctypes.data_as(_pi)

    def make_struct(self, sysd):
        keep = []
        s = OrcSystem()
        for name, ctype in OrcSystem._fields_:
            v = sysd.get(name)
            if ctype is _pd:
                if v is None:
                    v = np.zeros(1)
                a, p = self._d(v)
                keep.append(a)
                setattr(s, name, p)
            elif ctype is _pi:
                if v is None:
                    v = np.zeros(1, np.int32)
                a, p = self._i(v)
                keep.append(a)
                setattr(s, name, p)
            else:
                setattr(s, name, 0 if v is None else v)
        s._keep = keep
        return s

    # -- setup -------------------------------------------------------------
    def spline_table(self, nsplin, rmin, rmax, itype, sig, eps, alp, rheal, ishift):
        v = np.zeros(nsplin)
        dv = np.zeros(nsplin)
        dr = C.c_double()
        dri = C.c_double()
        self.lib.orc_spline_table(nsplin, rmin, rmax, itype, sig, eps, alp, rheal, ishift,
                                  v.ctypes.data_as(_pd), dv.ctypes.data_as(_pd), C.byref(dr), C.byref(dri))
        return v, dv, dr.value, dri.value

    def kvectors(self, kmax, hmat):
        hmat = np.ascontiguousarray(hmat, np.float64)
        hi = np.linalg.inv(hmat.reshape(3, 3, order="F")).reshape(-1, order="F")
        hi = np.ascontiguousarray(hi)
        deth = float(np.linalg.det(hmat.reshape(3, 3, order="F")))
        ecut = self.lib.orc_ewald_ecut(kmax, deth)
        kmaxv = np.zeros(3, np.int32)
        self.lib.orc_kmaxv(ecut, hi.ctypes.data_as(_pd), kmaxv.ctypes.data_as(_pi))
        n = self.lib.orc_kvec_count(ecut, kmaxv.ctypes.data_as(_pi), hi.ctypes.data_as(_pd))
        ka = np.zeros(n, np.int32)
        kb = np.zeros(n, np.int32)
        kc = np.zeros(n, np.int32)
        self.lib.orc_kvec_fill(ecut, kmaxv.ctypes.data_as(_pi), hi.ctypes.data_as(_pd),
                               ka.ctypes.data_as(_pi), kb.ctypes.data_as(_pi), kc.ctypes.data_as(_pi))
        return ecut, kmaxv, ka, kb, kc

    def pme_grid(self, ecut, hmat, kmaxv, kmax_pme):
        hmat = np.ascontiguousarray(hmat, np.float64)
        hi = np.ascontiguousarray(np.linalg.inv(hmat.reshape(3, 3, order="F")).reshape(-1, order="F"))
        deth = float(np.linalg.det(hmat.reshape(3, 3, order="F")))
        kmaxv = np.ascontiguousarray(kmaxv, np.int32)
        ng = np.zeros(3, np.int32)
        self.lib.orc_pme_grid(ecut, deth, hi.ctypes.data_as(_pd), kmaxv.ctypes.data_as(_pi), kmax_pme,
                              ng.ctypes.data_as(_pi))
        return ng

    def bweight(self, ka, kb, kc, ngrid, n_interp):
        ka, pa = self._i(ka)
        kb, pb = self._i(kb)
        kc, pc = self._i(kc)
        ng, pg = self._i(ngrid)
        bw = np.zeros(len(ka))
        self.lib.orc_pme_bweight(len(ka), pa, pb, pc, pg, n_interp, bw.ctypes.data_as(_pd))
        return bw

    def ecor_table(self, nsplin, rmax, alp, ecut):
        cv0 = np.zeros(nsplin)
        cdv0 = np.zeros(nsplin)
        dr = C.c_double()
        dri = C.c_double()
        se = C.c_double()
        self.lib.orc_ecor_table(nsplin, rmax, alp, ecut, cv0.ctypes.data_as(_pd), cdv0.ctypes.data_as(_pd),
                                C.byref(dr), C.byref(dri), C.byref(se))
        return cv0, cdv0, dr.value, dri.value, se.value

    def bond_power(self, c2, c3, c4):
        c = np.zeros(7)
        dc = np.zeros(7)
        self.lib.orc_bond_power(c2, c3, c4, c.ctypes.data_as(_pd), dc.ctypes.data_as(_pd))
        return c, dc

    def bend_harm(self, fk, theta0):
        out = [np.zeros(7) for _ in range(4)]
        self.lib.orc_bend_harm(fk, theta0, *[o.ctypes.data_as(_pd) for o in out])
        return out

    def clong(self, atm_typ, ntyp, c6, cutoff, rheal, iswit):
        at, pa = self._i(atm_typ)
        c6, p6 = self._d(c6)
        cu, pc = self._d(cutoff)
        return self.lib.orc_clong(len(at), ntyp, pa, p6, pc, rheal, iswit)

    # -- evaluation --------------------------------------------------------
    def check_list(self, pos, x0, skin, spread_ref, cutoff):
        """PINY's list rebuild test (orc_check_list): (rebuild, rmax,
        spread_now, cutskin2)."""
        pos = np.ascontiguousarray(pos, np.float64)
        P, natm = pos.shape[0], pos.shape[1]
        x0 = np.ascontiguousarray(x0, np.float64).reshape(natm, 3)
        cut = np.ascontiguousarray(cutoff, np.float64)
        cs = np.zeros(len(cut))
        rmax, sp = C.c_double(), C.c_double()
        f = self.lib.orc_check_list(natm, P, pos.ctypes.data_as(_pd), x0.ctypes.data_as(_pd), C.c_double(skin),
                                    C.c_double(spread_ref), len(cut), cut.ctypes.data_as(_pd), C.byref(rmax),
                                    C.byref(sp), cs.ctypes.data_as(_pd))
        return bool(f), rmax.value, sp.value, cs

    def pimd_transform(self, x, kind, what):
        """PINY's ring-polymer transform (orc_pimd_transform) of x[P][natm][3]:
        kind 1 staging / 2 normal modes; what 0 positions->modes,
        1 modes->positions, 2 forces->mode forces.  Returns a new array."""
        y = np.array(x, dtype=np.float64, order="C", copy=True)
        P, natm = y.shape[0], y.shape[1]
        rc = self.lib.orc_pimd_transform(natm, P, int(kind), int(what), y.ctypes.data_as(_pd))
        if rc != 0:
            raise ValueError("orc_pimd_transform: bad arguments")
        return y

    def verlist(self, sysd, pos1, xmod, hmat, cutskin2):
        s = self.make_struct(sysd)
        pos1 = np.ascontiguousarray(pos1, np.float64).reshape(-1, 3)
        x, y, z = [np.ascontiguousarray(pos1[:, d]) for d in range(3)]
        if xmod is not None:
            xm = np.ascontiguousarray(xmod, np.float64).reshape(-1, 3)
            xs = [np.ascontiguousarray(xm[:, d]) for d in range(3)]
            xp = [a.ctypes.data_as(_pd) for a in xs]
        else:
            xp = [None, None, None]
        hmat, ph = self._d(hmat)
        cs, pcs = self._d(cutskin2)
        n = sysd["natm"]
        cap = 0
        cnt = self.lib.orc_verlist(C.byref(s), x.ctypes.data_as(_pd), y.ctypes.data_as(_pd),
                                   z.ctypes.data_as(_pd), *xp, ph, None, pcs, cap, None, None)
        pi = np.zeros(max(cnt, 1), np.int32)
        pj = np.zeros(max(cnt, 1), np.int32)
        self.lib.orc_verlist(C.byref(s), x.ctypes.data_as(_pd), y.ctypes.data_as(_pd),
                             z.ctypes.data_as(_pd), *xp, ph, None, pcs, cnt,
                             pi.ctypes.data_as(_pi), pj.ctypes.data_as(_pi))
        del n
        return pi[:cnt], pj[:cnt]

    def verlist_rows(self, sysd, pos1, xmod, hmat, cutskin2, ilo, ihi):
        """The pairs (i, j) of verlist with ilo <= i < ihi."""
        s = self.make_struct(sysd)
        pos1 = np.ascontiguousarray(pos1, np.float64).reshape(-1, 3)
        xs = [np.ascontiguousarray(pos1[:, d]) for d in range(3)]
        xp = [a.ctypes.data_as(_pd) for a in xs]
        if xmod is not None:
            xm = np.ascontiguousarray(xmod, np.float64).reshape(-1, 3)
            ms = [np.ascontiguousarray(xm[:, d]) for d in range(3)]
            mp = [a.ctypes.data_as(_pd) for a in ms]
        else:
            mp = [None, None, None]
        hmat, ph = self._d(hmat)
        cs, pcs = self._d(cutskin2)
        cnt = self.lib.orc_verlist_rows(C.byref(s), *xp, *mp, ph, pcs, int(ilo), int(ihi), 0, None, None)
        pi = np.zeros(max(cnt, 1), np.int32)
        pj = np.zeros(max(cnt, 1), np.int32)
        self.lib.orc_verlist_rows(C.byref(s), *xp, *mp, ph, pcs, int(ilo), int(ihi), cnt,
                                  pi.ctypes.data_as(_pi), pj.ctypes.data_as(_pi))
        return pi[:cnt], pj[:cnt]

    def energy_force(self, sysd, pos, xmod, hmat, pi, pj, distribute_ghosts=False):
        s = self.make_struct(sysd)
        pos = np.ascontiguousarray(pos, np.float64)
        P = pos.shape[0]
        force = np.zeros_like(pos)
        xm = None
        if xmod is not None:
            xm = np.ascontiguousarray(xmod, np.float64)
        hmat, ph = self._d(hmat)
        pi, ppi = self._i(pi)
        pj, ppj = self._i(pj)
        e = OrcEnergies()
        self.lib.orc_energy_force(C.byref(s), P, pos.ctypes.data_as(_pd),
                                  xm.ctypes.data_as(_pd) if xm is not None else None, ph, len(pi),
                                  ppi, ppj, 1 if distribute_ghosts else 0, force.ctypes.data_as(_pd),
                                  C.byref(e))
        out = {n: getattr(e, n) for n, _ in OrcEnergies._fields_ if n != "pvten"}
        out["pvten"] = np.array(e.pvten[:])
        return force, out

    def respa_force(self, sysd, respa, level, pos, xmod, hmat, pi, pj, distribute_ghosts=False):
        """orc_respa_force: PINY's weighted forces at one RESPA level and, at
        a full inter level, the virial forces (else None).  ``respa`` holds
        wght_ter, wght_ter_res, wght_tra_res, int_res_ter, int_res_inter,
        ires_bond, cutoff_res [npair_typ], rheal_res, bond_eq_res and, for
        the reciprocal RESPA set, nktot_res, ecor_cdv0_res and (PINY's
        separate RESPA PME mesh) pme_res_on, ngrid_res, n_interp_res,
        kastr_res, kbstr_res, kcstr_res, bweight_res."""
        s = self.make_struct(sysd)
        r = OrcRespa()
        keep = []
        for name, ctype in OrcRespa._fields_:
            v = respa.get(name)
            if v is None:
                v = np.zeros(1) if ctype in (_pd, _pi) else (None if ctype is _i * 3 else 0)
            if ctype is _pd:
                a, p = self._d(v)
                keep.append(a)
                setattr(r, name, p)
            elif ctype is _pi:
                a, p = self._i(v)
                keep.append(a)
                setattr(r, name, p)
            elif ctype is _i * 3:
                if v is not None:
                    r.ngrid_res[:] = [int(x) for x in v]
            else:
                setattr(r, name, int(v) if ctype is _i else v)
        pos = np.ascontiguousarray(pos, np.float64)
        P = pos.shape[0]
        force = np.zeros_like(pos)
        forcet = np.zeros_like(pos)
        xm = None if xmod is None else np.ascontiguousarray(xmod, np.float64)
        hmat, ph = self._d(hmat)
        pi, ppi = self._i(pi)
        pj, ppj = self._i(pj)
        self.lib.orc_respa_force(C.byref(s), C.byref(r), int(level), P, pos.ctypes.data_as(_pd),
                                 xm.ctypes.data_as(_pd) if xm is not None else None, ph, len(pi), ppi, ppj,
                                 1 if distribute_ghosts else 0, force.ctypes.data_as(_pd),
                                 forcet.ctypes.data_as(_pd))
        del keep
        return force, (forcet if level & 1 else None)


# -- path-integral MD bookkeeping (pimd_oracle.c) and its composition -------

def _c(a, dt=np.float64):
    return np.ascontiguousarray(a, dt)


def nhc_apply(orc, v, m, chains, x_nhc, v_nhc):
    """apply_NHC_par on one bead's velocities v [natm][3] (copies returned)."""
    v, m = _c(v).copy(), _c(m)
    x_nhc, v_nhc = _c(x_nhc).copy(), _c(v_nhc).copy()
    inhc = _c(chains["inhc"], np.int32)
    w = _c(chains["wdti"])
    orc.lib.orc_nhc_apply(v.shape[0], inhc.ctypes.data_as(_pi), m.ctypes.data_as(_pd), v.ctypes.data_as(_pd),
                          int(chains["num_nhc"]), int(chains["len_nhc"]), int(chains["nres_nhc"]), len(w),
                          w.ctypes.data_as(_pd), _c(chains["mass_nhc"]).ctypes.data_as(_pd),
                          _c(chains["gkt"]).ctypes.data_as(_pd), x_nhc.ctypes.data_as(_pd), v_nhc.ctypes.data_as(_pd))
    return v, x_nhc, v_nhc


def pimd_springs(orc, u, prekf, veig, wght):
    """mode_energy_control: (fm, kin_harm, pvten_mode_tot)."""
    u = _c(u)
    fm = np.zeros_like(u)
    pv = np.zeros(9)
    prekf, veig = _c(prekf), _c(veig)
    ake = orc.lib.orc_pimd_springs(u.shape[1], u.shape[0], u.ctypes.data_as(_pd), prekf.ctypes.data_as(_pd),
                                   veig.ctypes.data_as(_pd), float(wght), fm.ctypes.data_as(_pd), pv.ctypes.data_as(_pd))
    return fm, ake, pv


def pimd_force_post(orc, kind, f, x, xmod, fm, nfree, beta, pvten, pvten_tot):
    """energy_control_pimd's post-processing: (mode forces, akvirx, pvten,
    pvten_tot)."""
    f = _c(f).copy()
    x, xmod, fm = _c(x), _c(xmod), _c(fm)
    pv, pvt = _c(pvten).copy(), _c(pvten_tot).copy()
    akv = orc.lib.orc_pimd_force_post(f.shape[1], f.shape[0], int(kind), f.ctypes.data_as(_pd), x.ctypes.data_as(_pd),
                                      xmod.ctypes.data_as(_pd), fm.ctypes.data_as(_pd), int(nfree), float(beta),
                                      pv.ctypes.data_as(_pd), pvt.ctypes.data_as(_pd))
    return f, akv, pv, pvt


def ghost_positions(sysd, x):
    """get_ghost_pos on every bead of x [P][natm][3] (a copy), in PINY's
    operation order: sum over components of coef * position."""
    x = _c(x).copy()
    ng = int(sysd.get("nghost", 0))
    if ng == 0:
        return x
    nc = int(sysd["ghost_ncomp"])
    comp = np.asarray(sysd["ghost_comp"]).reshape(ng, nc)
    coef = np.asarray(sysd["ghost_coef"], np.float64).reshape(ng, nc)
    acc = np.zeros((x.shape[0], ng, 3))
    for c in range(nc):
        ok = comp[:, c] >= 0
        term = coef[:, c][None, :, None] * x[:, np.where(ok, comp[:, c], 0), :]
        acc = np.where(ok[None, :, None], acc + term, acc)
    x[:, np.asarray(sysd["ghost_atom"]), :] = acc
    return x


def pimd_forces(orc, sysd, setup, x, pi, pj):
    """pinyb200_pimd_forces restated: (x with ghosts, mode forces, energies)."""
    P, kind = int(setup["nbeads"]), int(setup["kind"])
    x = ghost_positions(sysd, x)
    u = orc.pimd_transform(x, kind, 0) if P > 1 else x.copy()
    return (x,) + _forces_core(orc, sysd, setup, x, u, u[0].copy(), pi, pj)


def _forces_core(orc, sysd, setup, x, u, xmod, pi, pj):
    P, kind = int(setup["nbeads"]), int(setup["kind"])
    fm, ake, pvm = pimd_springs(orc, u, setup["prekf"], setup["path_eig"], setup.get("wght_pimd", 1.0))
    f, e = orc.energy_force(sysd, x, xmod if P > 1 else None, sysd["hmat"], pi, pj, distribute_ghosts=True)
    fmode, akv, pv, pvt = pimd_force_post(orc, kind, f, x, xmod, fm, setup["nfree_atoms"], setup["beta"],
                                          e["pvten"], e["pvten"])
    e = dict(e)
    e.update(kin_harm=ake, akvirx=akv if P > 1 else 0.0, pvten_corr=pv, pvten_tot_corr=pvt, pvten_mode_tot=pvm)
    return fmode, e


def pimd_apply_chains(orc, setup, v, state):
    """Class chains on bead 1 (atom masses), bead chains on beads 2..P."""
    v = _c(v).copy()
    cls, bead = setup.get("class_nhc"), setup.get("bead_nhc")
    if cls is not None and int(cls["num_nhc"]):
        v[0], state["cx"], state["cv"] = nhc_apply(orc, v[0], setup["mass"], cls, state["cx"], state["cv"])
    if bead is not None and int(bead["num_nhc"]):
        for b in range(1, v.shape[0]):
            v[b], state["bx"][b - 1], state["bv"][b - 1] = nhc_apply(orc, v[b], setup["bead_mass"][b], bead,
                                                                     state["bx"][b - 1], state["bv"][b - 1])
    return v


def pimd_force_post_respa(orc, kind, f, ft, x, xmod, fm, nfree, beta, full, pvten, pvten_tot):
    """energy_control_pimd's post-processing at one RESPA level: (mode
    forces, akvirx, pvten, pvten_tot); ft = the virial forces (full level)."""
    f = _c(f).copy()
    ftc = None if ft is None else _c(ft).copy()
    x, xmod, fm = _c(x), _c(xmod), _c(fm)
    pv, pvt = _c(pvten).copy(), _c(pvten_tot).copy()
    akv = orc.lib.orc_pimd_force_post_respa(f.shape[1], f.shape[0], int(kind), f.ctypes.data_as(_pd),
                                            None if ftc is None else ftc.ctypes.data_as(_pd), x.ctypes.data_as(_pd),
                                            xmod.ctypes.data_as(_pd), fm.ctypes.data_as(_pd), int(nfree), float(beta),
                                            1 if full else 0, pv.ctypes.data_as(_pd), pvt.ctypes.data_as(_pd))
    return f, akv, pv, pvt


def pimd_forces_respa(orc, sysd, setup, respa, x, pi, pj):
    """pinyb200_pimd_forces with RESPA counts > 1: the outer level, as
    PINY's first force call (control_pimd.c:297-317).  Returns (x with
    ghosts, mode forces, energies)."""
    P, kind = int(setup["nbeads"]), int(setup["kind"])
    x = ghost_positions(sysd, x)
    u = orc.pimd_transform(x, kind, 0) if P > 1 else x.copy()
    xmod = u[0].copy()
    fm, ake, pvm = pimd_springs(orc, u, setup["prekf"], setup["path_eig"], setup.get("wght_pimd", 1.0))
    level = 1 | 4 | 8 | (2 if respa["int_res_ter"] else 0)
    fw, ft = orc.respa_force(sysd, respa, level, x, xmod if P > 1 else None, sysd["hmat"], pi, pj,
                             distribute_ghosts=True)
    _, ef = orc.energy_force(sysd, x, xmod if P > 1 else None, sysd["hmat"], pi, pj, distribute_ghosts=True)
    f, akv, pv, pvt = pimd_force_post_respa(orc, kind, fw, ft, x, xmod, fm, setup["nfree_atoms"], setup["beta"],
                                            True, ef["pvten"], ef["pvten"])
    e = dict(ef)
    e.update(kin_harm=ake, akvirx=akv if P > 1 else 0.0, pvten_tot_corr=pvt, pvten_mode_tot=pvm)
    return x, f, e


def pimd_step_respa(orc, sysd, setup, respa, x, v, f, state, pi, pj):
    """pinyb200_pimd_step with RESPA counts setup["nres"] = (nres_ter,
    nres_tor, nres_tra, nres_pimd) and chains at level setup["ix_respa"]:
    int_NVT_pimd's nested loops (int_NVT_pimd.c:142-223) with
    int_0_to_dt2_nvt_pimd / int_dt2_to_dt_nvt_pimd (int_0_to_dt2_pimd.c:
    34-190, int_dt2_to_dt_pimd.c) and the force path at each level
    (orc_respa_force, then orc_pimd_force_post_respa).  Returns new (x, v,
    f, energies of the outer level); `state` is updated."""
    P, kind, dt = int(setup["nbeads"]), int(setup["kind"]), float(setup["dt"])
    nt, no, na, npi = (int(k) for k in setup["nres"])
    ixr = int(setup.get("ix_respa", 1))
    dti = dt / float(nt * no * na * npi)
    bm = np.asarray(setup["bead_mass"], np.float64)[:, :, None]
    x, v, f = _c(x).copy(), _c(v).copy(), _c(f).copy()
    u = None
    e = None
    for ir_ter in range(1, nt + 1):
        for ir_tor in range(1, no + 1):
            for ir_tra in range(1, na + 1):
                for ir_pimd in range(1, npi + 1):
                    ix = 5
                    if ir_pimd == 1:
                        ix = 4
                        if ir_tra == 1:
                            ix = 3
                            if ir_tor == 1:
                                ix = 1 if ir_ter == 1 else 2
                    if ixr >= ix:
                        v = pimd_apply_chains(orc, setup, v, state)
                    v = v + (f * (dti / 2.0)) / bm
                    if ir_pimd == 1:
                        u = orc.pimd_transform(x, kind, 0) if P > 1 else x.copy()
                    u = u + v * dti
                    fm, ake, pvm = pimd_springs(orc, u, setup["prekf"], setup["path_eig"], setup.get("wght_pimd", 1.0))
                    if ir_pimd == npi:
                        xmod = u[0].copy()
                        x = orc.pimd_transform(u, kind, 1) if P > 1 else u.copy()
                        x = ghost_positions(sysd, x)
                        last_tra = ir_tra == na
                        level = 8 | (4 if last_tra else 0)
                        if respa["int_res_ter"] and ir_tor == no and last_tra:
                            level |= 2
                        full = ir_ter == nt and ir_tor == no and last_tra
                        if full:
                            level |= 1
                        fw, ft = orc.respa_force(sysd, respa, level, x, xmod if P > 1 else None, sysd["hmat"], pi, pj,
                                                 distribute_ghosts=True)
                        if full:
                            _, ef = orc.energy_force(sysd, x, xmod if P > 1 else None, sysd["hmat"], pi, pj,
                                                     distribute_ghosts=True)
                            pv0 = ef["pvten"]
                        else:
                            pv0 = np.zeros(9)
                        f, akv, pv, pvt = pimd_force_post_respa(orc, kind, fw, ft, x, xmod, fm, setup["nfree_atoms"],
                                                                setup["beta"], full, pv0, pv0)
                        if full:
                            e = dict(ef)
                            e.update(kin_harm=ake, akvirx=akv if P > 1 else 0.0, pvten_tot_corr=pvt,
                                     pvten_mode_tot=pvm)
                    else:
                        f = fm
                    v = v + (f * (dti / 2.0)) / bm
                    ix = 5
                    if ir_pimd == npi:
                        ix = 4
                        if ir_tra == na:
                            ix = 3
                            if ir_tor == no:
                                ix = 1 if ir_ter == nt else 2
                    if ixr >= ix:
                        v = pimd_apply_chains(orc, setup, v, state)
    return x, v, f, e


def pimd_step(orc, sysd, setup, x, v, f, state, pi, pj):
    """pinyb200_pimd_step restated (int_NVT_pimd with RESPA counts 1):
    returns new (x, v, f, energies); `state` (chain x/v) is updated."""
    P, kind, dt = int(setup["nbeads"]), int(setup["kind"]), float(setup["dt"])
    bm = np.asarray(setup["bead_mass"], np.float64)[:, :, None]
    v = pimd_apply_chains(orc, setup, v, state)
    v = v + (f * (dt / 2.0)) / bm
    u = orc.pimd_transform(x, kind, 0) if P > 1 else _c(x).copy()
    u = u + v * dt
    xmod = u[0].copy()
    xn = orc.pimd_transform(u, kind, 1) if P > 1 else u.copy()
    xn = ghost_positions(sysd, xn)
    fn, e = _forces_core(orc, sysd, setup, xn, u, xmod, pi, pj)
    v = v + (fn * (dt / 2.0)) / bm
    v = pimd_apply_chains(orc, setup, v, state)
    return xn, v, fn, e
