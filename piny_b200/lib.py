"""ctypes binding of the pinyb200 C ABI (include/pinyb200.h).

The device library is the only compute path: if libpinyb200.so is missing
and cannot be built, or no GPU is present, every call raises.  There is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

_i = C.c_int
_d = C.c_double
_pi = C.POINTER(C.c_int)
_pd = C.POINTER(C.c_double)

PINYB200_FP64 = 0
PINYB200_MIXED = 1
DISTRIB_GHOSTS = 1
NO_ENERGY = 2
SITE_PAIRS = 4
TUNE_AGAIN = 8
UPDATE_LIST = 16       # PINYB200_UPDATE_LIST
BATCH_BRANCHES = 32    # PINYB200_BATCH_BRANCHES
BATCH_KERNELS = 64     # PINYB200_BATCH_KERNELS

STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_NO_DEVICE", 4: "ERR_LIST_OVERFLOW", 5: "ERR_CUTOFF",
          6: "ERR_TIMEOUT", 7: "ERR_NAN", 8: "ERR_UNSUPPORTED", 9: "ERR_STATE"}


class PinySystem(C.Structure):
    """pinyb200_system (include/pinyb200.h)."""
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


ENERGY_NAMES = ("vreal", "vvdw", "vcoul", "vrecip", "vself", "vbgr", "vecor", "vlong",
                "vbond", "vbend", "vintert", "vintrat")


class PinyEnergies(C.Structure):
    _fields_ = [(n, _d) for n in ENERGY_NAMES] + [("pvten", _d * 9)]


class PinyListState(C.Structure):
    """pinyb200_list_state."""
    _fields_ = [("rebuilds", C.c_long), ("rebuilt_last", _i), ("overflow", _i), ("mismatch", _i), ("rmax", _d),
                ("spread_now", _d), ("spread_ref", _d), ("npairs", C.c_long), ("nactive", C.c_long),
                ("nmol_pairs", C.c_long)]


class PinyNhcSet(C.Structure):
    """pinyb200_nhc_set: one Nose-Hoover chain set (PINY THERM_INFO)."""
    _fields_ = [("num_nhc", _i), ("len_nhc", _i), ("nres_nhc", _i), ("nyosh_nhc", _i), ("wdti", _pd), ("inhc", _pi),
                ("mass_nhc", _pd), ("gkt", _pd)]


class PinyPimdSetup(C.Structure):
    """pinyb200_pimd_setup."""
    _fields_ = [("natm", _i), ("nbeads", _i), ("kind", _i), ("mass", _pd), ("bead_mass", _pd), ("prekf", _pd),
                ("path_eig", _pd), ("wght_pimd", _d), ("dt", _d), ("beta", _d), ("nfree_atoms", _i),
                ("class_nhc", PinyNhcSet), ("bead_nhc", PinyNhcSet),
                ("nres_ter", _i), ("nres_tor", _i), ("nres_tra", _i), ("nres_pimd", _i), ("ix_respa", _i)]


class PinyPimdEnergies(C.Structure):
    """pinyb200_pimd_energies."""
    _fields_ = [("force", PinyEnergies), ("kin_harm", _d), ("akvirx", _d), ("pvten", _d * 9), ("pvten_tot", _d * 9),
                ("pvten_mode_tot", _d * 9)]


class PinyRespa(C.Structure):
    _fields_ = [("wght_ter", _d), ("wght_ter_res", _d), ("wght_tra_res", _d),
                ("int_res_ter", _i), ("int_res_inter", _i), ("ires_bond", _i),
                ("cutoff_res", _pd), ("rheal_res", _d), ("bond_eq_res", _pd), ("nktot_res", _i),
                ("pme_res_on", _i), ("ecor_cdv0_res", _pd), ("ngrid_res", _i * 3), ("n_interp_res", _i),
                ("kastr_res", _pi), ("kbstr_res", _pi), ("kcstr_res", _pi), ("bweight_res", _pd)]


class PinyTangent(C.Structure):
    """pinyb200_tangent: derivative of the set-up data along one parameter."""
    _fields_ = [("dcharge", _pd), ("dcv0", _pd), ("dcdv0", _pd), ("dghost_coef", _pd), ("dbond_eq", _pd),
                ("dbond_c", _pd), ("dbend_c", _pd), ("dbend_s", _pd), ("dbend_dc", _pd), ("dbend_ds", _pd),
                ("dclong", _d)]


# every symbol include/pinyb200.h declares
EXPORTS = ("pinyb200_version", "pinyb200_device_info", "pinyb200_create", "pinyb200_destroy",
           "pinyb200_build_list", "pinyb200_get_list", "pinyb200_list_info", "pinyb200_energy_force",
           "pinyb200_energy_force_device", "pinyb200_piny_force", "pinyb200_last_timing",
           "pinyb200_last_error", "pinyb200_count_list_device", "pinyb200_check_list_device",
           "pinyb200_autotune", "pinyb200_get_tuning", "pinyb200_set_tuning", "pinyb200_batch_create",
           "pinyb200_batch_destroy", "pinyb200_batch_energy_force_device", "pinyb200_batch_last_ms",
           "pinyb200_batch_last_error", "pinyb200_batch_last_mode", "pinyb200_grad_prepare", "pinyb200_grad",
           "pinyb200_fma_peak", "pinyb200_pimd_transform", "pinyb200_pimd_create", "pinyb200_pimd_destroy",
           "pinyb200_pimd_set_nhc", "pinyb200_pimd_get_nhc", "pinyb200_pimd_forces", "pinyb200_pimd_step",
           "pinyb200_update_list_device", "pinyb200_list_set_spread", "pinyb200_list_status",
           "pinyb200_set_respa", "pinyb200_respa_force_device", "pinyb200_piny_force_respa",
           "pinyb200_set_kernel_timing", "pinyb200_kernel_times", "pinyb200_set_list_method",
           "pinyb200_list_cells")

LIST_LNK, LIST_NOLST = 0, 1                       # PINYB200_LIST_LNK / _NOLST
STAGING, NORMAL_MODES = 1, 2                      # PINYB200_STAGING / _NORMAL_MODES
TO_MODES, TO_BEADS, FORCE_TO_MODES = 0, 1, 2      # PINYB200_TO_MODES / _TO_BEADS / _FORCE_TO_MODES

COUNT_MAX_ATOMS = 65536       # PINYB200_COUNT_MAX_ATOMS
COUNT_MAX_PAIR_TYPES = 64     # PINYB200_COUNT_MAX_PAIR_TYPES

_LIB = None


class PinyError(RuntimeError):
    pass


def load(build_if_missing: bool = True):
    """Load (building if needed) the in-tree libpinyb200.so."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = _build.LIB
    if not os.path.exists(path) or (build_if_missing and _build.needs_build()):
        if not build_if_missing:
            raise PinyError("libpinyb200.so is not built (python -m piny_b200.build)")
        _build.build()
    L = C.CDLL(path)
    L.pinyb200_version.restype = _i
    L.pinyb200_device_info.argtypes = [C.c_char_p, _i, _pi]
    L.pinyb200_create.argtypes = [C.POINTER(PinySystem), _i, _i, C.POINTER(C.c_void_p)]
    L.pinyb200_destroy.argtypes = [C.c_void_p]
    L.pinyb200_build_list.argtypes = [C.c_void_p, _pd, _pd, _pd, _pd, C.POINTER(C.c_long)]
    L.pinyb200_get_list.argtypes = [C.c_void_p, _pi, _pi, C.c_long, C.POINTER(C.c_long)]
    L.pinyb200_set_list_method.argtypes = [C.c_void_p, _i]
    L.pinyb200_list_cells.argtypes = [C.c_void_p, _pi]
    L.pinyb200_list_info.argtypes = [C.c_void_p, C.POINTER(C.c_long), C.POINTER(C.c_long), C.POINTER(C.c_long)]
    L.pinyb200_energy_force.argtypes = [C.c_void_p, _pd, _pd, _pd, _i, _pd, C.POINTER(PinyEnergies)]
    L.pinyb200_energy_force_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _pd, _i, C.c_void_p,
                                               C.POINTER(PinyEnergies), C.c_void_p]
    L.pinyb200_piny_force.argtypes = [C.c_void_p] + [C.c_void_p] * 3 + [_pd] * 3 + [_pd] + [C.c_void_p] * 3 + \
        [_pd, C.POINTER(PinyEnergies)]
    L.pinyb200_last_timing.argtypes = [C.c_void_p, C.POINTER(C.c_float), _i]
    L.pinyb200_set_kernel_timing.argtypes = [C.c_void_p, _i]
    L.pinyb200_kernel_times.argtypes = [C.c_void_p, C.POINTER(C.c_char_p), C.POINTER(C.c_float), _i,
                                        C.POINTER(C.c_int)]
    L.pinyb200_count_list_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _pd, _pd, C.POINTER(C.c_long),
                                             C.POINTER(C.c_long), C.c_void_p]
    L.pinyb200_check_list_device.argtypes = [C.c_void_p, C.c_void_p, _d, _pi, _pd, _pd, _pd, C.c_void_p]
    L.pinyb200_autotune.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _pd, _i, _i, _pi, C.POINTER(C.c_float)]
    L.pinyb200_get_tuning.argtypes = [C.c_void_p, _pi]
    L.pinyb200_set_tuning.argtypes = [C.c_void_p, _pi]
    L.pinyb200_batch_create.argtypes = [C.POINTER(C.c_void_p), _i, C.POINTER(C.c_void_p)]
    L.pinyb200_batch_destroy.argtypes = [C.c_void_p]
    L.pinyb200_batch_energy_force_device.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                                     C.POINTER(_pd), _i, C.POINTER(C.c_void_p),
                                                     C.POINTER(PinyEnergies), C.c_void_p]
    L.pinyb200_batch_last_ms.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
    L.pinyb200_batch_last_mode.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.pinyb200_batch_last_error.restype = C.c_char_p
    L.pinyb200_batch_last_error.argtypes = [C.c_void_p]
    L.pinyb200_grad_prepare.argtypes = [C.c_void_p, _i, C.POINTER(PinyTangent)]
    L.pinyb200_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _pd, C.c_void_p, _pd, _pd, C.c_void_p]
    L.pinyb200_fma_peak.argtypes = [_i, _i, _pd]
    L.pinyb200_pimd_transform.argtypes = [_i, _i, _i, _i, C.c_void_p, C.c_void_p]
    L.pinyb200_update_list_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _pd, C.c_void_p]
    L.pinyb200_list_set_spread.argtypes = [C.c_void_p, _d]
    L.pinyb200_list_status.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(PinyListState)]
    L.pinyb200_pimd_create.argtypes = [C.POINTER(PinyPimdSetup), C.POINTER(C.c_void_p)]
    L.pinyb200_pimd_destroy.argtypes = [C.c_void_p]
    L.pinyb200_pimd_set_nhc.argtypes = [C.c_void_p, _i, _pd, _pd]
    L.pinyb200_pimd_get_nhc.argtypes = [C.c_void_p, _i, _pd, _pd]
    L.pinyb200_pimd_forces.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, _pd,
                                       C.POINTER(PinyPimdEnergies), C.c_void_p]
    L.pinyb200_pimd_step.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, _pd,
                                     C.POINTER(PinyPimdEnergies), C.c_void_p]
    L.pinyb200_last_error.restype = C.c_char_p
    L.pinyb200_set_respa.argtypes = [C.c_void_p, C.POINTER(PinyRespa)]
    L.pinyb200_respa_force_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _pd, _i, _i, C.c_void_p,
                                              C.c_void_p, C.POINTER(PinyEnergies), C.c_void_p]
    L.pinyb200_piny_force_respa.argtypes = [C.c_void_p, _i] + [C.c_void_p] * 3 + [_pd] * 3 + [_pd] + \
        [C.c_void_p] * 6 + [_pd, C.POINTER(PinyEnergies)]
    L.pinyb200_last_error.argtypes = [C.c_void_p]
    _LIB = L
    return L


def fma_peak_gflops(fp64=False, reps=5):
    """Measured FMA throughput of the current GPU (GFLOP/s)."""
    L = load()
    g = C.c_double()
    rc = L.pinyb200_fma_peak(1 if fp64 else 0, int(reps), C.byref(g))
    if rc != 0:
        raise PinyError("pinyb200_fma_peak: %s %s" % (STATUS.get(rc, rc), L.pinyb200_last_error(None).decode()))
    return g.value


def pimd_transform(d_x, natm, nbeads, kind, what, stream=None):
    """PINY's ring-polymer transform (staging or normal modes), in place on
    the device array at address d_x, shaped [nbeads][natm][3] FP64:
    what TO_MODES (positions -> modes), TO_BEADS (modes -> positions) or
    FORCE_TO_MODES (bead forces -> mode forces).  Enqueued on `stream`
    (a CUDA stream handle; None for the default stream)."""
    L = load()
    rc = L.pinyb200_pimd_transform(int(natm), int(nbeads), int(kind), int(what), C.c_void_p(d_x),
                                   C.c_void_p(stream) if stream else None)
    if rc != 0:
        raise PinyError("pinyb200_pimd_transform: %s %s" % (STATUS.get(rc, rc), L.pinyb200_last_error(None).decode()))


def _dp(a):
    return a.ctypes.data_as(_pd)


def make_struct(sysd: dict):
    """pinyb200_system from a set-up dict (piny_b200.system.build_system)."""
    keep = []
    s = PinySystem()
    for name, ctype in PinySystem._fields_:
        v = sysd.get(name)
        if ctype is _pd:
            a = np.ascontiguousarray(np.zeros(1) if v is None else v, dtype=np.float64)
            keep.append(a)
            setattr(s, name, a.ctypes.data_as(_pd))
        elif ctype is _pi:
            a = np.ascontiguousarray(np.zeros(1, np.int32) if v is None else v, dtype=np.int32)
            keep.append(a)
            setattr(s, name, a.ctypes.data_as(_pi))
        else:
            setattr(s, name, 0 if v is None else v)
    s._keep = keep
    return s


def energies_dict(e: PinyEnergies):
    out = {n: getattr(e, n) for n in ENERGY_NAMES}
    out["pvten"] = np.array(e.pvten[:])
    return out


class DeviceBox:
    """One box of nbeads beads resident on the GPU (a pinyb200 context)."""

    def __init__(self, sysd: dict, nbeads: int, precision: str = "fp64"):
        self.L = load()
        self.natm = int(sysd["natm"])
        self.P = int(nbeads)
        self.ntyp = int(sysd["ntyp"])
        self.precision = precision
        prec = PINYB200_FP64 if precision == "fp64" else PINYB200_MIXED
        st = make_struct(sysd)
        h = C.c_void_p()
        rc = self.L.pinyb200_create(C.byref(st), self.P, prec, C.byref(h))
        if rc != 0:
            raise PinyError("pinyb200_create: %s %s" % (STATUS.get(rc, rc), self.L.pinyb200_last_error(None).decode()))
        self.h = h

    def _check(self, rc, what):
        if rc != 0:
            raise PinyError("%s: %s %s" % (what, STATUS.get(rc, rc), self.L.pinyb200_last_error(self.h).decode()))

    def close(self):
        if getattr(self, "h", None):
            self.L.pinyb200_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build_list(self, pos1, xmod, hmat, cutskin2):
        pos1 = np.ascontiguousarray(pos1, np.float64).reshape(self.natm, 3)
        xm = None if xmod is None else np.ascontiguousarray(xmod, np.float64).reshape(self.natm, 3)
        hmat = np.ascontiguousarray(hmat, np.float64)
        cs = np.ascontiguousarray(cutskin2, np.float64)
        n = C.c_long()
        self._check(self.L.pinyb200_build_list(self.h, _dp(pos1), None if xm is None else _dp(xm), _dp(hmat),
                                               _dp(cs), C.byref(n)), "build_list")
        return n.value

    def count_list_device(self, d_pos1: int, d_xmod, hmat, cutskin2, stream=None):
        """Pair counts (npairs, nactive) for device-resident bead-1 positions,
        through the allocation-free pinyb200_count_list_device."""
        hmat = np.ascontiguousarray(hmat, np.float64)
        cs = np.ascontiguousarray(cutskin2, np.float64)
        n, a = C.c_long(), C.c_long()
        self._check(self.L.pinyb200_count_list_device(self.h, C.c_void_p(d_pos1),
                                                      None if d_xmod is None else C.c_void_p(d_xmod), _dp(hmat),
                                                      _dp(cs), C.byref(n), C.byref(a),
                                                      None if stream is None else C.c_void_p(stream)),
                    "count_list_device")
        return n.value, a.value

    def check_list_device(self, d_pos: int, spread_ref: float = 0.0, stream=None):
        """PINY's list rebuild test for device-resident positions [P][natm][3]:
        (rebuild, rmax, spread_now, cutskin2 for the next build)."""
        reb = C.c_int()
        rmax, spread = C.c_double(), C.c_double()
        cs = np.zeros(self.ntyp * (self.ntyp + 1) // 2)
        self._check(self.L.pinyb200_check_list_device(self.h, C.c_void_p(d_pos), float(spread_ref), C.byref(reb),
                                                      C.byref(rmax), C.byref(spread), _dp(cs),
                                                      None if stream is None else C.c_void_p(stream)),
                    "check_list_device")
        return bool(reb.value), rmax.value, spread.value, cs

    def update_list_device(self, d_pos: int, d_xmod, hmat, stream=None):
        """PINY's list test and, when due, rebuild on the device (no host
        round trip); d_pos [P][natm][3] with current ghost positions."""
        hm = np.ascontiguousarray(hmat, np.float64)
        self._check(self.L.pinyb200_update_list_device(self.h, C.c_void_p(d_pos),
                                                       C.c_void_p(d_xmod) if d_xmod else None, _dp(hm),
                                                       C.c_void_p(stream) if stream else None),
                    "update_list_device")

    def list_set_spread(self, spread_ref: float):
        self._check(self.L.pinyb200_list_set_spread(self.h, float(spread_ref)), "list_set_spread")

    def list_status(self, stream=None, check=True):
        st = PinyListState()
        rc = self.L.pinyb200_list_status(self.h, C.c_void_p(stream) if stream else None, C.byref(st))
        if check:
            self._check(rc, "list_status")
        return {k: getattr(st, k) for k, _ in PinyListState._fields_}

    def get_list(self):
        n = C.c_long()
        self._check(self.L.pinyb200_get_list(self.h, None, None, 0, C.byref(n)), "get_list")
        pi = np.zeros(max(n.value, 1), np.int32)
        pj = np.zeros(max(n.value, 1), np.int32)
        self._check(self.L.pinyb200_get_list(self.h, pi.ctypes.data_as(_pi), pj.ctypes.data_as(_pi), n.value,
                                             C.byref(n)), "get_list")
        return pi[:n.value], pj[:n.value]

    def set_list_method(self, method):
        """LIST_LNK (link cells when the box allows, the default) or LIST_NOLST (all-pairs sweep)."""
        self._check(self.L.pinyb200_set_list_method(self.h, int(method)), "set_list_method")

    def list_cells(self):
        """Cells along a, b, c of the current list's plan (zeros: swept) and whether the cells built it."""
        cells = np.zeros(4, np.int32)
        self._check(self.L.pinyb200_list_cells(self.h, cells.ctypes.data_as(_pi)), "list_cells")
        return tuple(int(v) for v in cells[:3]), bool(cells[3])

    def list_info(self):
        n, a, c = C.c_long(), C.c_long(), C.c_long()
        self._check(self.L.pinyb200_list_info(self.h, C.byref(n), C.byref(a), C.byref(c)), "list_info")
        return {"npairs": n.value, "nactive": a.value, "capacity": c.value}

    def energy_force(self, pos, xmod, hmat, distribute_ghosts=False, energy=True, site_pairs=False):
        pos = np.ascontiguousarray(pos, np.float64).reshape(self.P, self.natm, 3)
        xm = None if xmod is None else np.ascontiguousarray(xmod, np.float64).reshape(self.natm, 3)
        hmat = np.ascontiguousarray(hmat, np.float64)
        force = np.empty_like(pos)
        e = PinyEnergies()
        flags = (DISTRIB_GHOSTS if distribute_ghosts else 0) | (0 if energy else NO_ENERGY) | \
            (SITE_PAIRS if site_pairs else 0)
        self._check(self.L.pinyb200_energy_force(self.h, _dp(pos), None if xm is None else _dp(xm), _dp(hmat),
                                                 flags, _dp(force), C.byref(e)), "energy_force")
        return force, energies_dict(e)

    def energy_force_device(self, d_pos: int, d_xmod, hmat, d_force: int, stream=None, distribute_ghosts=False,
                            energy=True, update_list=False):
        """Device-pointer variant; pointers are integers (e.g. tensor.data_ptr()).
        update_list: PINY's list test and rebuild on the device first."""
        hmat = np.ascontiguousarray(hmat, np.float64)
        e = PinyEnergies()
        flags = (DISTRIB_GHOSTS if distribute_ghosts else 0) | (0 if energy else NO_ENERGY) | \
            (UPDATE_LIST if update_list else 0)
        self._check(self.L.pinyb200_energy_force_device(self.h, C.c_void_p(d_pos),
                                                        None if d_xmod is None else C.c_void_p(d_xmod), _dp(hmat),
                                                        flags, C.c_void_p(d_force), C.byref(e),
                                                        None if stream is None else C.c_void_p(stream)),
                    "energy_force_device")
        return energies_dict(e)

    def set_respa(self, respa):
        """PINY's RESPA split (a dict as piny_b200.respa.respa_setup makes;
        None switches it off)."""
        if respa is None:
            self._check(self.L.pinyb200_set_respa(self.h, None), "set_respa")
            return
        cut = np.ascontiguousarray(respa["cutoff_res"], np.float64)
        eqr = np.ascontiguousarray(respa["bond_eq_res"], np.float64)
        ecr = respa.get("ecor_cdv0_res")
        ecr = None if ecr is None else np.ascontiguousarray(ecr, np.float64)
        r = PinyRespa(float(respa["wght_ter"]), float(respa["wght_ter_res"]), float(respa["wght_tra_res"]),
                      int(respa["int_res_ter"]), int(respa["int_res_inter"]), int(respa["ires_bond"]), _dp(cut),
                      float(respa["rheal_res"]), _dp(eqr), int(respa.get("nktot_res", 0)),
                      int(respa.get("pme_res_on", 0)), None if ecr is None else _dp(ecr))
        keep = []
        if int(respa.get("pme_res_on", 0)) and "ngrid_res" in respa:
            # PINY's separate RESPA PME mesh: its size, order, k sphere and weights
            r.ngrid_res[:] = [int(v) for v in respa["ngrid_res"]]
            r.n_interp_res = int(respa["n_interp_res"])
            for name in ("kastr_res", "kbstr_res", "kcstr_res"):
                a = np.ascontiguousarray(respa[name], np.int32)
                keep.append(a)
                setattr(r, name, a.ctypes.data_as(_pi))
            bw = np.ascontiguousarray(respa["bweight_res"], np.float64)
            keep.append(bw)
            r.bweight_res = _dp(bw)
        self._check(self.L.pinyb200_set_respa(self.h, C.byref(r)), "set_respa")

    def respa_force_device(self, d_pos: int, d_xmod, hmat, level: int, d_force: int, d_forcet=None, stream=None,
                           distribute_ghosts=False, energy=True, update_list=False):
        """One RESPA level (piny_b200.respa bits) from device positions:
        PINY's weighted forces into d_force and, at the outer level, the
        unweighted virial forces into d_forcet; returns the energies (zero
        at inner levels)."""
        hmat = np.ascontiguousarray(hmat, np.float64)
        e = PinyEnergies()
        flags = (DISTRIB_GHOSTS if distribute_ghosts else 0) | (0 if energy else NO_ENERGY) | \
            (UPDATE_LIST if update_list else 0)
        self._check(self.L.pinyb200_respa_force_device(self.h, C.c_void_p(d_pos),
                                                       None if d_xmod is None else C.c_void_p(d_xmod), _dp(hmat),
                                                       int(level), flags, C.c_void_p(d_force),
                                                       None if d_forcet is None else C.c_void_p(d_forcet),
                                                       C.byref(e), None if stream is None else C.c_void_p(stream)),
                    "respa_force_device")
        return energies_dict(e)

    def autotune(self, d_pos: int, d_xmod, hmat, reps=3, again=False, energy=True):
        """Time every launch shape on these inputs and keep the fastest:
        returns (choice [tile, pair kernel, blocks/SM, overlap], best ms or -1
        when a remembered result was applied)."""
        hmat = np.ascontiguousarray(hmat, np.float64)
        ch = (C.c_int * 4)()
        ms = C.c_float()
        flags = (TUNE_AGAIN if again else 0) | (0 if energy else NO_ENERGY)
        self._check(self.L.pinyb200_autotune(self.h, C.c_void_p(d_pos), None if d_xmod is None else C.c_void_p(d_xmod),
                                             _dp(hmat), flags, int(reps), ch, C.byref(ms)), "autotune")
        return list(ch), ms.value

    def tuning(self):
        ch = (C.c_int * 4)()
        self._check(self.L.pinyb200_get_tuning(self.h, ch), "get_tuning")
        return list(ch)

    def set_tuning(self, choice):
        ch = (C.c_int * 4)(*[int(v) for v in choice])
        self._check(self.L.pinyb200_set_tuning(self.h, ch), "set_tuning")

    def grad_prepare(self, tangents):
        """Upload tangent channels: a list of dicts with keys of PinyTangent
        (arrays or scalars; missing keys are zero)."""
        arr = (PinyTangent * max(1, len(tangents)))()
        keep = []
        for k, t in enumerate(tangents):
            for name, ctype in PinyTangent._fields_:
                v = t.get(name)
                if ctype is _pd:
                    if v is None:
                        setattr(arr[k], name, None)
                    else:
                        a = np.ascontiguousarray(v, np.float64)
                        keep.append(a)
                        setattr(arr[k], name, _dp(a))
                else:
                    setattr(arr[k], name, float(v or 0.0))
        self._check(self.L.pinyb200_grad_prepare(self.h, len(tangents), arr), "grad_prepare")
        self._ntan = len(tangents)

    def grad(self, d_pos: int, d_xmod, hmat, d_fbar=None, stream=None):
        """(dE, dF) per prepared tangent (see pinyb200_grad)."""
        hmat = np.ascontiguousarray(hmat, np.float64)
        n = max(1, getattr(self, "_ntan", 0))
        dE = np.zeros(n)
        dF = np.zeros(n)
        self._check(self.L.pinyb200_grad(self.h, C.c_void_p(d_pos), None if d_xmod is None else C.c_void_p(d_xmod),
                                         _dp(hmat), None if d_fbar is None else C.c_void_p(d_fbar), _dp(dE), _dp(dF),
                                         None if stream is None else C.c_void_p(stream)), "grad")
        k = getattr(self, "_ntan", 0)
        return dE[:k], dF[:k]

    def set_kernel_timing(self, on=True):
        """Serialised evaluations with an event after every kernel."""
        self._check(self.L.pinyb200_set_kernel_timing(self.h, 1 if on else 0), "set_kernel_timing")

    def kernel_times(self):
        """[(kernel, ms)] of the last evaluation, in launch order."""
        names = (C.c_char_p * 64)()
        ms = (C.c_float * 64)()
        n = C.c_int()
        self._check(self.L.pinyb200_kernel_times(self.h, names, ms, 64, C.byref(n)), "kernel_times")
        return [(names[i].decode(), float(ms[i])) for i in range(n.value)]

    def last_timing(self):
        ms = (C.c_float * 5)()
        self._check(self.L.pinyb200_last_timing(self.h, ms, 5), "last_timing")
        return list(ms)


class DeviceBatch:
    """Several DeviceBox contexts evaluated together as one CUDA graph launch
    (pinyb200_batch_*)."""

    def __init__(self, boxes):
        self.L = load()
        self.boxes = list(boxes)
        arr = (C.c_void_p * len(self.boxes))(*[b.h.value for b in self.boxes])
        h = C.c_void_p()
        rc = self.L.pinyb200_batch_create(arr, len(self.boxes), C.byref(h))
        if rc != 0:
            raise PinyError("pinyb200_batch_create: %s %s" % (STATUS.get(rc, rc),
                                                              self.L.pinyb200_last_error(None).decode()))
        self.h = h

    def energy_force_device(self, d_pos, d_xmod, hmats, d_force, stream=None, energy=True, update_list=False,
                            branches=False, kernels=False, distribute_ghosts=False):
        """Every box in one graph launch: the faster of the multi-box kernels
        and one graph branch per box (timed at capture) where the kernels
        cover the boxes, else branches; kernels=True / branches=True pick one."""
        n = len(self.boxes)
        P = (C.c_void_p * n)(*[int(p) for p in d_pos])
        X = (C.c_void_p * n)(*[None if x is None else int(x) for x in d_xmod]) if d_xmod is not None else None
        F = (C.c_void_p * n)(*[int(p) for p in d_force])
        hm = [np.ascontiguousarray(h, np.float64) for h in hmats]
        H = (_pd * n)(*[_dp(h) for h in hm])
        E = (PinyEnergies * n)()
        flags = (0 if energy else NO_ENERGY) | (UPDATE_LIST if update_list else 0) | \
            (BATCH_BRANCHES if branches else 0) | (BATCH_KERNELS if kernels else 0) | \
            (DISTRIB_GHOSTS if distribute_ghosts else 0)
        rc = self.L.pinyb200_batch_energy_force_device(self.h, P, X, H, flags, F, E,
                                                       None if stream is None else C.c_void_p(stream))
        if rc != 0:
            raise PinyError("batch_energy_force_device: %s %s" % (STATUS.get(rc, rc),
                                                                  self.L.pinyb200_batch_last_error(self.h).decode()))
        return [energies_dict(e) for e in E]

    def last_ms(self):
        ms = C.c_float()
        self.L.pinyb200_batch_last_ms(self.h, C.byref(ms))
        return ms.value

    def tune(self, d_pos, d_xmod, hmats, d_force, stream=None, reps=3):
        """Launch shapes for the batch as a whole: each box's own autotuned
        shape (pinyb200_autotune, timed on the box alone), the default
        shapes, and the defaults with each box's own PME tile edge are each
        timed as a batch call (the capture keeps the faster graph form for
        each); the fastest set is kept.  Returns {set name: ms} and the kept
        set's name."""
        base = [b.tuning() for b in self.boxes]
        own = [b.autotune(d_pos[i], None if d_xmod is None else d_xmod[i], hmats[i], reps=2)[0]
               for i, b in enumerate(self.boxes)]
        times = {}
        # the defaults with each box's own PME tile edge: the tile choice
        # alone, without the per-box pair-kernel choices
        tiles = [[o[0]] + list(d[1:]) for o, d in zip(own, base)]
        sets = {"per_box": own, "defaults": base, "defaults_own_tiles": tiles}
        for name, choice in sets.items():
            for b, ch in zip(self.boxes, choice):
                b.set_tuning(ch)
            ts = []
            for k in range(reps + 1):
                self.energy_force_device(d_pos, d_xmod, hmats, d_force, stream=stream)
                if k:
                    ts.append(self.last_ms())
            times[name] = float(np.median(ts))
        keep = min(times, key=times.get)
        for b, ch in zip(self.boxes, sets[keep]):
            b.set_tuning(ch)
        return times, keep

    def last_mode(self):
        """(fused, kernel launches) of the graph the last call ran."""
        f, k = C.c_int(), C.c_int()
        self.L.pinyb200_batch_last_mode(self.h, C.byref(f), C.byref(k))
        return bool(f.value), int(k.value)

    def close(self):
        if getattr(self, "h", None):
            self.L.pinyb200_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _pimd_energies(e):
    out = {k: getattr(e.force, k) for k in ENERGY_NAMES}
    out["force_pvten"] = np.array(e.force.pvten[:])
    out["kin_harm"] = e.kin_harm
    out["akvirx"] = e.akvirx
    for k in ("pvten", "pvten_tot", "pvten_mode_tot"):
        out[k] = np.array(getattr(e, k)[:])
    return out


class DevicePimd:
    """PINY's NVT ring-polymer step on the device (pinyb200_pimd_*), driving
    the force path of a DeviceBox.  `setup` holds the numpy arrays of
    pinyb200_pimd_setup (see piny_b200.pimd.nvt_setup)."""

    def __init__(self, setup: dict):
        self.L = load()
        self._keep = []
        self.natm, self.P = int(setup["natm"]), int(setup["nbeads"])

        def dp(a, dt=np.float64):
            a = np.ascontiguousarray(a, dt)
            self._keep.append(a)
            return a.ctypes.data_as(_pd if dt == np.float64 else _pi)

        def nhc(c):
            if c is None or int(c["num_nhc"]) == 0:
                return PinyNhcSet(0, 0, 0, 0, None, None, None, None)
            return PinyNhcSet(int(c["num_nhc"]), int(c["len_nhc"]), int(c["nres_nhc"]), len(c["wdti"]),
                              dp(c["wdti"]), dp(c["inhc"], np.int32), dp(c["mass_nhc"]), dp(c["gkt"]))

        self.sets = (setup.get("class_nhc"), setup.get("bead_nhc"))
        st = PinyPimdSetup(self.natm, self.P, int(setup["kind"]), dp(setup["mass"]), dp(setup["bead_mass"]),
                           dp(setup["prekf"]), dp(setup["path_eig"]), float(setup.get("wght_pimd", 1.0)),
                           float(setup["dt"]), float(setup["beta"]), int(setup["nfree_atoms"]),
                           nhc(self.sets[0]), nhc(self.sets[1]), *[int(v) for v in setup.get("nres", (1, 1, 1, 1))],
                           int(setup.get("ix_respa", 1)))
        h = C.c_void_p()
        self._check(self.L.pinyb200_pimd_create(C.byref(st), C.byref(h)), "pinyb200_pimd_create")
        self.h = h

    def _check(self, rc, what):
        if rc != 0:
            raise PinyError("%s: %s %s" % (what, STATUS.get(rc, rc), self.L.pinyb200_last_error(None).decode()))

    def _shape(self, s):
        c = self.sets[s]
        if c is None or int(c["num_nhc"]) == 0:
            return None
        nb = 1 if s == 0 else self.P - 1
        return (nb, int(c["len_nhc"]), int(c["num_nhc"])) if s == 1 else (int(c["len_nhc"]), int(c["num_nhc"]))

    def set_nhc(self, s, x_nhc, v_nhc):
        if self._shape(s) is None:
            return
        x = np.ascontiguousarray(x_nhc, np.float64).reshape(self._shape(s))
        v = np.ascontiguousarray(v_nhc, np.float64).reshape(self._shape(s))
        self._check(self.L.pinyb200_pimd_set_nhc(self.h, s, _dp(x), _dp(v)), "pinyb200_pimd_set_nhc")

    def get_nhc(self, s):
        shp = self._shape(s)
        if shp is None:
            return None, None
        x, v = np.zeros(shp), np.zeros(shp)
        self._check(self.L.pinyb200_pimd_get_nhc(self.h, s, _dp(x), _dp(v)), "pinyb200_pimd_get_nhc")
        return x, v

    def forces(self, box, d_x, d_f, hmat, stream=None):
        hm = np.ascontiguousarray(hmat, np.float64)
        e = PinyPimdEnergies()
        self._check(self.L.pinyb200_pimd_forces(self.h, box.h, C.c_void_p(d_x), C.c_void_p(d_f), _dp(hm),
                                                C.byref(e), C.c_void_p(stream) if stream else None),
                    "pinyb200_pimd_forces")
        return _pimd_energies(e)

    def step(self, box, d_x, d_v, d_f, hmat, stream=None):
        hm = np.ascontiguousarray(hmat, np.float64)
        e = PinyPimdEnergies()
        self._check(self.L.pinyb200_pimd_step(self.h, box.h, C.c_void_p(d_x), C.c_void_p(d_v), C.c_void_p(d_f),
                                              _dp(hm), C.byref(e), C.c_void_p(stream) if stream else None),
                    "pinyb200_pimd_step")
        return _pimd_energies(e)

    def close(self):
        if getattr(self, "h", None):
            self.L.pinyb200_pimd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
