"""RESPA split on the device against PINY's forces at each RESPA level
(golden fixtures from ``piny_ref respa``) and against the oracle
restatement on seeded inputs.

Tolerances (force relative RMS): FP64 1e-12, MIXED 1e-5.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import RESPA_NAMES, fixture_level, load_fixture, pair_hash, respa_from_fixture, rel_rms

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "mixed": 1e-5}
ETOL = {"fp64": 1e-11, "mixed": 1e-6}


def _dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, np.float64), device="cuda")


def _levels(box, F, prec, pos, xmod, hmat, distribute=False):
    """Forces of the four levels int_NVT_pimd sets, the outer level's virial
    forces and energies."""
    import torch
    d_pos = _dev(pos)
    d_xm = None if xmod is None else _dev(xmod)
    out = []
    ft = torch.zeros_like(d_pos)
    e0 = None
    for lv in range(4):
        f = torch.zeros_like(d_pos)
        e = box.respa_force_device(d_pos.data_ptr(), None if d_xm is None else d_xm.data_ptr(), hmat,
                                   fixture_level(F, lv), f.data_ptr(), ft.data_ptr() if lv == 0 else None,
                                   distribute_ghosts=distribute)
        out.append(f.cpu().numpy())
        if lv == 0:
            e0 = e
    return out, ft.cpu().numpy(), e0


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", RESPA_NAMES)
def test_respa_levels_match_piny(name, prec):
    from piny_b200.lib import DeviceBox
    F = load_fixture(name)
    box = DeviceBox(F, int(F["nbeads"]), prec)
    xmod = F.get("xmod")
    box.build_list(F["pos"][0], xmod, F["hmat"], F["cutskin2"])
    gi, gj = box.get_list()
    assert pair_hash(gi, gj) == F["pairs_sha256"]
    box.set_respa(respa_from_fixture(F))
    forces, ft, e0 = _levels(box, F, prec, F["pos"], xmod, F["hmat"])
    for lv in range(4):
        assert rel_rms(forces[lv], F["ref_L%d_force_raw" % lv]) < TOL[prec], lv
    if "ref_L0_forcet_raw" in F:
        assert rel_rms(ft, F["ref_L0_forcet_raw"]) < TOL[prec]
    # the outer level's energies are the plain evaluation's
    _, e = box.energy_force(F["pos"], xmod, F["hmat"])
    for k in ("vintert", "vintrat", "vrecip", "vecor", "vbond", "vbend"):
        assert abs(e0[k] - e[k]) <= ETOL[prec] * max(1.0, abs(e[k])), k
    assert np.abs(e0["pvten"] - e["pvten"]).max() <= ETOL[prec] * 10 * np.abs(e["pvten"]).max()
    box.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_respa_matches_oracle_seeded(prec, oracle):
    """q-TIP4P/F 128 molecules, P = 2, moved off the list positions (as
    between rebuilds), a RESPA set-up of step counts (3, 1, 2, 2) and ghosts
    distributed; every level against the oracle."""
    from piny_b200.lib import DeviceBox
    from piny_b200 import respa as R
    F = load_fixture("tip4pf_128_p2")
    xmod = F["xmod"]
    pi, pj = oracle.verlist(F, F["pos"][0], xmod, F["hmat"], F["cutskin2"])
    rng = np.random.default_rng(7)
    pos = F["pos"] + rng.uniform(-0.05, 0.05, F["pos"].shape)
    rs = R.respa_setup(3, 1, 2, 2, True, True, np.asarray(F["cutoff"]) - 2.0, 1.4,
                       np.asarray(F["bond_eq"]) + 0.03)
    box = DeviceBox(F, 2, prec)
    box.build_list(F["pos"][0], xmod, F["hmat"], F["cutskin2"])
    box.set_respa(rs)
    import torch
    d_pos, d_xm = _dev(pos), _dev(xmod)
    for lv in R.loop_levels(3, 1, 2, 2, True):
        if lv == 0:
            continue
        fref, ftref = oracle.respa_force(F, rs, lv, pos, xmod, F["hmat"], pi, pj, distribute_ghosts=True)
        f = torch.zeros_like(d_pos)
        ft = torch.zeros_like(d_pos)
        box.respa_force_device(d_pos.data_ptr(), d_xm.data_ptr(), F["hmat"], lv, f.data_ptr(), ft.data_ptr(),
                               distribute_ghosts=True)
        assert rel_rms(f.cpu().numpy(), fref) < TOL[prec], lv
        if ftref is not None:
            assert rel_rms(ft.cpu().numpy(), ftref) < TOL[prec]
    box.close()


def test_respa_arguments():
    from piny_b200.lib import DeviceBox, PinyError
    from piny_b200 import respa as R
    F = load_fixture("respa_spcfw_64_p1")
    box = DeviceBox(F, 1, "fp64")
    box.build_list(F["pos"][0], None, F["hmat"], F["cutskin2"])
    import torch
    d_pos = _dev(F["pos"])
    f = torch.zeros_like(d_pos)
    with pytest.raises(PinyError, match="ERR_STATE"):
        box.respa_force_device(d_pos.data_ptr(), None, F["hmat"], R.RES_INTRA, f.data_ptr())
    rs = respa_from_fixture(F)
    bad = dict(rs, cutoff_res=np.asarray(F["cutoff"]) + 1.0)
    with pytest.raises(PinyError, match="ERR_ARG"):
        box.set_respa(bad)
    with pytest.raises(PinyError, match="ERR_ARG"):
        box.set_respa(dict(rs, nktot_res=12, pme_res_on=1))  # the RESPA mesh's k sphere is needed
    G = load_fixture("respa_pmegrid_tip4pf_64_p4")
    mesh = respa_from_fixture(G)
    with pytest.raises(PinyError, match="ERR_UNSUPPORTED"):
        box.set_respa(dict(rs, nktot_res=mesh["nktot_res"], pme_res_on=1, ngrid_res=mesh["ngrid_res"],
                           n_interp_res=12, kastr_res=mesh["kastr_res"], kbstr_res=mesh["kbstr_res"],
                           kcstr_res=mesh["kcstr_res"], bweight_res=mesh["bweight_res"],
                           ecor_cdv0_res=G["ecor_cdv0_res"]))
    with pytest.raises(PinyError, match="ERR_ARG"):
        box.set_respa(dict(rs, nktot_res=12))  # the RESPA exclusion table is needed
    box.set_respa(rs)
    # levels PINY's loops never set are refused
    for lv in (R.FULL_INTER, R.RES_INTER, R.FULL_INTER | R.FULL_INTRA | R.RES_INTRA):
        with pytest.raises(PinyError, match="ERR_ARG"):
            box.respa_force_device(d_pos.data_ptr(), None, F["hmat"], lv, f.data_ptr())
    # PINY's first call sets RES_INTRA only with intra RESPA: same forces
    f2 = torch.zeros_like(d_pos)
    box.respa_force_device(d_pos.data_ptr(), None, F["hmat"], R.FULL_INTER | R.RES_INTER | R.FULL_INTRA, f.data_ptr())
    box.respa_force_device(d_pos.data_ptr(), None, F["hmat"], R.FULL_INTER | R.RES_INTER | R.FULL_INTRA | R.RES_INTRA,
                           f2.data_ptr())
    assert rel_rms(f.cpu().numpy(), f2.cpu().numpy()) < 1e-13  # up to the atomics' summation order
    box.set_respa(dict(rs, int_res_ter=0))
    with pytest.raises(PinyError, match="ERR_ARG"):
        box.respa_force_device(d_pos.data_ptr(), None, F["hmat"], R.RES_INTER | R.FULL_INTRA | R.RES_INTRA,
                               f.data_ptr())
    box.close()


def _piny_arrays(a):
    """PINY's per-bead 1-based arrays (double*[P]) for a [P][natm] array."""
    P, n = a.shape
    bufs = [np.zeros(n + 1) for _ in range(P)]
    for b in range(P):
        bufs[b][1:] = a[b]
    ptrs = (C.c_void_p * P)(*[x.ctypes.data for x in bufs])
    return bufs, ptrs


def test_piny_layout_calls():
    """The PINY-layout entry points add to PINY's 1-based per-bead arrays:
    the plain call as pinyb200_energy_force, the RESPA call as the device
    call, with the virial forces at the outer level."""
    from piny_b200.lib import DeviceBox, PinyEnergies
    F = load_fixture("respa_tip4pf_64_p4")
    P, n = int(F["nbeads"]), int(F["natm"])
    box = DeviceBox(F, P, "fp64")
    xmod = F["xmod"]
    box.build_list(F["pos"][0], xmod, F["hmat"], F["cutskin2"])
    box.set_respa(respa_from_fixture(F))
    pos = F["pos"]
    keep = []
    X = []
    for d in range(3):
        bufs, ptrs = _piny_arrays(pos[:, :, d])
        keep.append(bufs)
        X.append(ptrs)
    xm = [np.concatenate([[0.0], xmod[:, d]]) for d in range(3)]
    h1 = np.concatenate([[0.0], np.asarray(F["hmat"], np.float64)])
    seed = np.random.default_rng(3).normal(size=(3, P, n))
    Fa, Ft = [], []
    for d in range(3):
        bufs, ptrs = _piny_arrays(seed[d])
        keep.append(bufs)
        Fa.append((bufs, ptrs))
        bufs2, ptrs2 = _piny_arrays(np.zeros((P, n)))
        keep.append(bufs2)
        Ft.append((bufs2, ptrs2))
    pv = np.zeros(10)
    e = PinyEnergies()
    dp = C.POINTER(C.c_double)
    rc = box.L.pinyb200_piny_force_respa(box.h, fixture_level(F, 0), X[0], X[1], X[2],
                                          *[a.ctypes.data_as(dp) for a in xm], h1.ctypes.data_as(dp),
                                          Fa[0][1], Fa[1][1], Fa[2][1], Ft[0][1], Ft[1][1], Ft[2][1],
                                          pv.ctypes.data_as(dp), C.byref(e))
    assert rc == 0
    got = np.stack([np.stack([Fa[d][0][b][1:] for b in range(P)]) for d in range(3)], axis=-1)
    want = F["ref_L0_force_raw"] + np.moveaxis(seed, 0, -1)
    assert rel_rms(got, want) < 1e-12
    gt = np.stack([np.stack([Ft[d][0][b][1:] for b in range(P)]) for d in range(3)], axis=-1)
    assert rel_rms(gt, F["ref_L0_forcet_raw"]) < 1e-12
    # an inner level adds its weighted forces and leaves the virial forces
    for d in range(3):
        for b in range(P):
            Fa[d][0][b][:] = 0.0
    before = [[Ft[d][0][b].copy() for b in range(P)] for d in range(3)]
    rc = box.L.pinyb200_piny_force_respa(box.h, fixture_level(F, 1), X[0], X[1], X[2],
                                          *[a.ctypes.data_as(dp) for a in xm], h1.ctypes.data_as(dp),
                                          Fa[0][1], Fa[1][1], Fa[2][1], Ft[0][1], Ft[1][1], Ft[2][1],
                                          None, C.byref(e))
    assert rc == 0
    got = np.stack([np.stack([Fa[d][0][b][1:] for b in range(P)]) for d in range(3)], axis=-1)
    assert rel_rms(got, F["ref_L1_force_raw"]) < 1e-12
    assert all(np.array_equal(Ft[d][0][b], before[d][b]) for d in range(3) for b in range(P))
    # plain PINY-layout call: the unweighted forces, added to zeros
    for d in range(3):
        for b in range(P):
            Ft[d][0][b][:] = 0.0
    pv2 = np.zeros(10)
    rc = box.L.pinyb200_piny_force(box.h, X[0], X[1], X[2], *[a.ctypes.data_as(dp) for a in xm],
                                   h1.ctypes.data_as(dp), Ft[0][1], Ft[1][1], Ft[2][1], pv2.ctypes.data_as(dp),
                                   C.byref(e))
    assert rc == 0
    gt = np.stack([np.stack([Ft[d][0][b][1:] for b in range(P)]) for d in range(3)], axis=-1)
    assert rel_rms(gt, F["ref_L0_forcet_raw"]) < 1e-12
    assert np.abs(pv2[1:] - pv[1:]).max() <= 1e-12 * np.abs(pv[1:]).max()
    box.close()


@pytest.mark.parametrize("prec", ["fp64"])
def test_respa_list_follows_device_rebuild(prec, oracle):
    """A list rebuild on the device (PINYB200_UPDATE_LIST) rebuilds the RESPA
    pair list with it: after the atoms move past the skin, the inner and
    outer levels match the oracle on a list built afresh."""
    import torch

    from piny_b200 import respa as R
    from piny_b200.lib import DeviceBox
    F = load_fixture("tip4pf_128_p2")
    P, n = int(F["nbeads"]), int(F["natm"])
    rs = R.respa_setup(2, 1, 1, 1, True, True, np.asarray(F["cutoff"]) - 1.5, 1.2, np.asarray(F["bond_eq"]))
    box = DeviceBox(F, P, prec)
    box.build_list(F["pos"][0], F["xmod"], F["hmat"], F["cutskin2"])
    box.set_respa(rs)
    d0 = _dev(F["pos"])
    box.list_set_spread(box.check_list_device(d0.data_ptr(), 0.0)[2])
    rng = np.random.default_rng(11)
    nsite = 4  # q-TIP4P/F: O, H, H, M; molecules move rigidly
    shift = rng.normal(size=(n // nsite, 3))
    shift *= (0.7 * float(F["skin"]) / np.linalg.norm(shift, axis=1))[:, None]
    pos = F["pos"] + np.repeat(shift, nsite, axis=0)[None, :, :]
    xmod = pos.mean(axis=0)
    d_pos, d_xm = _dev(pos), _dev(xmod)
    inner = R.RES_INTER | R.FULL_INTRA | R.RES_INTRA
    f = torch.zeros_like(d_pos)
    box.respa_force_device(d_pos.data_ptr(), d_xm.data_ptr(), F["hmat"], inner, f.data_ptr(), update_list=True)
    st = box.list_status()
    assert st["rebuilds"] == 1 and not st["overflow"]
    cs = np.asarray(F["cutskin2"])
    pi, pj = oracle.verlist(F, pos[0], xmod, F["hmat"], cs)
    fref, _ = oracle.respa_force(F, rs, inner, pos, xmod, F["hmat"], pi, pj)
    assert rel_rms(f.cpu().numpy(), fref) < TOL[prec]
    outer = R.FULL_INTER | R.RES_INTER | R.FULL_INTRA | R.RES_INTRA
    ft = torch.zeros_like(d_pos)
    box.respa_force_device(d_pos.data_ptr(), d_xm.data_ptr(), F["hmat"], outer, f.data_ptr(), ft.data_ptr())
    fref, ftref = oracle.respa_force(F, rs, outer, pos, xmod, F["hmat"], pi, pj)
    assert rel_rms(f.cpu().numpy(), fref) < TOL[prec]
    assert rel_rms(ft.cpu().numpy(), ftref) < TOL[prec]
    box.close()
