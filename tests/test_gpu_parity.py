"""Device path against PINY's outputs (golden fixtures) and the oracle.

Tolerances (force relative RMS  ||F - F_ref|| / ||F_ref||):
  FP64 mode   1e-12
  MIXED mode  1e-5
Pair sets must match PINY's bit for bit in every mode.
"""
import numpy as np
import pytest

from helpers import GOLDEN_NAMES, load_fixture, pair_hash, rel_rms

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "mixed": 1e-5}
ETOL = {"fp64": 1e-11, "mixed": 1e-6}


def _box(F, prec):
    from piny_b200.lib import DeviceBox
    return DeviceBox(F, int(F["nbeads"]), prec)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_device_matches_piny(name, prec):
    F = load_fixture(name)
    box = _box(F, prec)
    xmod = F.get("xmod")
    n = box.build_list(F["pos"][0], xmod, F["hmat"], F["cutskin2"])
    pi, pj = box.get_list()
    assert n == F["npairs"]
    assert pair_hash(pi, pj) == F["pairs_sha256"]
    force, e = box.energy_force(F["pos"], xmod, F["hmat"])
    assert rel_rms(force, F["ref_force_raw"]) < TOL[prec]
    force2, _ = box.energy_force(F["pos"], xmod, F["hmat"], distribute_ghosts=True)
    assert rel_rms(force2, F["ref_force"]) < TOL[prec]
    # the site-list kernel (general fallback) agrees as well
    force3, e3 = box.energy_force(F["pos"], xmod, F["hmat"], site_pairs=True)
    assert rel_rms(force3, F["ref_force_raw"]) < TOL[prec]
    assert abs(e3["vintert"] - e["vintert"]) <= ETOL[prec] * max(1.0, abs(e["vintert"]))
    for k, kr in [("vintert", "vintert"), ("vintrat", "vintrat"), ("vvdw", "vvdw"), ("vcoul", "vcoul"),
                  ("vlong", "vlong"), ("vbond", "vbondt"), ("vbend", "vbendt")]:
        ref = F["ref_" + kr]
        assert abs(e[k] - ref) <= ETOL[prec] * max(1.0, abs(ref)), (k, e[k], ref)
    vrec = e["vrecip"] + e["vself"] + e["vbgr"] + e["vecor"]
    assert abs(vrec - F["ref_vrecip"]) <= ETOL[prec] * max(1.0, abs(F["ref_vrecip"]))
    pv = F["ref_pvten_tot"]
    assert np.abs(e["pvten"] - pv).max() <= ETOL[prec] * 10 * np.abs(pv).max()
    box.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_device_matches_oracle_32_beads(prec, oracle):
    """q-SPC/Fw 256 molecules, P = 32 (mixed-precision config), host set-up
    from piny_b200.system, oracle on the same inputs."""
    from piny_b200 import system, water
    spec = water.named_spec("spcfw_256_p32")
    pos = water.build_positions(spec) / water.BOHR
    S = system.build_system(spec, pos)
    xmod = pos.mean(axis=0)
    pi, pj = oracle.verlist(S, pos[0], xmod, S["hmat"], S["cutskin2"])
    fref, eref = oracle.energy_force(S, pos, xmod, S["hmat"], pi, pj)
    from piny_b200.lib import DeviceBox
    box = DeviceBox(S, spec.nbeads, prec)
    n = box.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
    gi, gj = box.get_list()
    assert n == len(pi) and pair_hash(gi, gj) == pair_hash(pi, pj)
    f, e = box.energy_force(pos, xmod, S["hmat"])
    assert rel_rms(f, fref) < TOL[prec]
    assert abs(e["vintert"] - eref["vintert"]) <= ETOL[prec] * abs(eref["vintert"])
    assert abs(e["vintrat"] - eref["vintrat"]) <= ETOL[prec] * abs(eref["vintrat"])
    box.close()


def test_list_errors_and_state():
    F = load_fixture("spcfw_64_p1")
    from piny_b200.lib import DeviceBox, PinyError
    box = DeviceBox(F, 1, "fp64")
    with pytest.raises(PinyError, match="ERR_STATE"):
        box.energy_force(F["pos"], None, F["hmat"])
    box.close()
    bad = dict(F)
    bad["atm_typ"] = np.array(F["atm_typ"]) + 5
    with pytest.raises(PinyError, match="ERR_ARG"):
        DeviceBox(bad, 1, "fp64")
    with pytest.raises(PinyError, match="ERR_UNSUPPORTED"):
        DeviceBox(F, 3, "fp64")


def _grid_case(case):
    """Systems that reach each PME FFT path: compile-time 64^3 and 128^3
    grids, and a non-cubic grid with a non-power-of-two edge (run-time path
    with the direct DFT)."""
    import dataclasses

    from piny_b200 import system, water
    if case == "tip4pf_512_g64":
        spec = water.BoxSpec(water.TIP4P_F, 512, water.density_box_edge(512), 2, 298.0, 99, grid=64, order=8)
    elif case == "spcfw_216_g128":
        spec = water.BoxSpec(water.SPC_FW, 216, 18.64, 1, 300.0, 5, grid=128, order=8)
    else:
        spec = dataclasses.replace(water.named_spec("spcfw_216_p4"), nbeads=2)
    pos = water.build_positions(spec) / water.BOHR
    S = system.build_system(spec, pos)
    if case == "spcfw_216_ncubic":
        # stretch the c axis of the mesh to 40 points, B-spline weights to match
        nc = 40
        wa = system.bspline_weight_1d(spec.order, S["ngrid_a"])
        wb = system.bspline_weight_1d(spec.order, S["ngrid_b"])
        wc = system.bspline_weight_1d(spec.order, nc)
        ka, kb, kc = S["kastr"], S["kbstr"], S["kcstr"]
        S["ngrid_c"] = nc
        S["bweight"] = wa[np.where(ka < 0, ka + S["ngrid_a"], ka)] * wb[np.where(kb < 0, kb + S["ngrid_b"], kb)] \
            * wc[np.where(kc < 0, kc + nc, kc)]
    return spec, pos, S


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["tip4pf_512_g64", "spcfw_216_g128", "spcfw_216_ncubic"])
def test_pme_grid_paths_match_oracle(case, prec, oracle):
    spec, pos, S = _grid_case(case)
    from piny_b200.lib import DeviceBox, PinyError
    if case == "spcfw_216_g128" and prec == "fp64":
        # an FP64 plane of 128 x 129 complex points exceeds shared memory
        with pytest.raises(PinyError, match="ERR_UNSUPPORTED"):
            DeviceBox(S, spec.nbeads, prec)
        return
    xmod = pos.mean(axis=0) if spec.nbeads > 1 else None
    pi, pj = oracle.verlist(S, pos[0], xmod, S["hmat"], S["cutskin2"])
    fref, eref = oracle.energy_force(S, pos, xmod, S["hmat"], pi, pj)
    box = DeviceBox(S, spec.nbeads, prec)
    box.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
    f, e = box.energy_force(pos, xmod, S["hmat"])
    assert rel_rms(f, fref) < TOL[prec]
    # both sums are small differences of large terms: their mixed-precision
    # error scales with the terms, not with the difference
    vrec = e["vrecip"] + e["vself"] + e["vbgr"] + e["vecor"]
    vrec_ref = eref["vrecip"] + eref["vself"] + eref["vbgr"] + eref["vecor"]
    rscale = abs(eref["vrecip"]) + abs(eref["vself"]) + abs(eref["vbgr"]) + abs(eref["vecor"])
    assert abs(vrec - vrec_ref) <= ETOL[prec] * max(1.0, rscale)
    scale = abs(eref["vvdw"]) + abs(eref["vcoul"]) + abs(eref["vrecip"]) + abs(eref["vself"]) + abs(eref["vecor"])
    assert abs(e["vintert"] - eref["vintert"]) <= ETOL[prec] * scale
    box.close()


@pytest.mark.parametrize("name", ["tip4pf_64_p4", "spcfw_64_p1"])
def test_list_check_matches_oracle(name, oracle):
    """Device rebuild test (check_ver_list + get_pimd_spread + get_cut_skin)
    against the oracle, bit for bit, before and after a displacement."""
    import torch

    from piny_b200.lib import DeviceBox
    F = load_fixture(name)
    P = int(F["nbeads"])
    box = DeviceBox(F, P, "fp64")
    xmod = F.get("xmod")
    pos = np.ascontiguousarray(F["pos"], np.float64)
    box.build_list(pos[0], xmod, F["hmat"], F["cutskin2"])
    x0 = pos[0].copy()
    rng = np.random.default_rng(11)
    cutoff = np.asarray(F["cutoff"], np.float64)
    skin = float(F["skin"])
    for scale, spread_ref in ((0.0, 0.0), (0.2, 0.1), (1.5, 0.0)):
        p = pos + rng.normal(scale=scale, size=pos.shape) if scale else pos
        d = torch.from_numpy(np.ascontiguousarray(p)).to("cuda:0")
        torch.cuda.synchronize()
        reb, rmax, sp, cs = box.check_list_device(d.data_ptr(), spread_ref)
        f, r_o, s_o, cs_o = oracle.check_list(p, x0, skin, spread_ref, cutoff)
        assert (reb, rmax, sp) == (f, r_o, s_o)
        assert np.array_equal(cs, cs_o)
    box.close()


def test_non_finite_positions_are_reported():
    """A NaN position gives PINYB200_ERR_NAN from the host-buffer call (the
    device work itself runs on the NaN and finishes normally)."""
    F = load_fixture("spcfw_64_p1")
    from piny_b200.lib import DeviceBox, PinyError
    box = DeviceBox(F, 1, "fp64")
    box.build_list(F["pos"][0], None, F["hmat"], F["cutskin2"])
    pos = np.array(F["pos"], np.float64)
    pos[0, 5, 1] = np.nan
    with pytest.raises(PinyError, match="ERR_NAN"):
        box.energy_force(pos, None, F["hmat"])
    # the context stays usable
    force, e = box.energy_force(F["pos"], None, F["hmat"])
    assert np.isfinite(e["vintert"])
    box.close()


def _oracle_case(oracle, spec, S, pos):
    xmod = pos.mean(axis=0) if spec.nbeads > 1 else None
    pi, pj = oracle.verlist(S, pos[0], xmod, S["hmat"], S["cutskin2"])
    fref, eref = oracle.energy_force(S, pos, xmod, S["hmat"], pi, pj)
    return xmod, pi, pj, fref, eref


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["triclinic", "beads64", "uncharged"])
def test_more_systems_match_oracle(case, prec, oracle):
    """A sheared (triclinic) cell: the site-list kernel, general minimum
    image and general-cell PME; 64 beads; a system without charges (no
    PME, no Ewald correction)."""
    import dataclasses

    from piny_b200 import system, water
    from piny_b200.lib import DeviceBox
    if case == "triclinic":
        spec = dataclasses.replace(water.named_spec("spcfw_216_p4"), nbeads=2)
        pos = water.build_positions(spec) / water.BOHR
        L = spec.L / water.BOHR
        h = np.array([L, 0.0, 0.0, 0.12 * L, L, 0.0, -0.07 * L, 0.05 * L, L])
        S = system.build_system(spec, pos, hmat=h)
    elif case == "beads64":
        spec = water.BoxSpec(water.TIP4P_F, 64, water.density_box_edge(64), 64, 298.0, 8, grid=16, order=8)
        pos = water.build_positions(spec) / water.BOHR
        S = system.build_system(spec, pos)
    else:
        model = dataclasses.replace(water.SPC_FW, charges=[0.0, 0.0, 0.0])
        spec = water.BoxSpec(model, 216, 18.64, 2, 300.0, 12, grid=32, order=6)
        pos = water.build_positions(spec) / water.BOHR
        S = system.build_system(spec, pos)
    xmod, pi, pj, fref, eref = _oracle_case(oracle, spec, S, pos)
    box = DeviceBox(S, spec.nbeads, prec)
    n = box.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
    gi, gj = box.get_list()
    assert n == len(pi) and pair_hash(gi, gj) == pair_hash(pi, pj)
    f, e = box.energy_force(pos, xmod, S["hmat"])
    assert rel_rms(f, fref) < TOL[prec]
    scale = abs(eref["vvdw"]) + abs(eref["vcoul"]) + abs(eref["vrecip"]) + abs(eref["vself"]) + abs(eref["vecor"])
    assert abs(e["vintert"] - eref["vintert"]) <= ETOL[prec] * max(scale, 1.0)
    assert abs(e["vintrat"] - eref["vintrat"]) <= ETOL[prec] * max(1.0, abs(eref["vintrat"]))
    box.close()
