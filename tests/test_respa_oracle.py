"""The RESPA split: the oracle restatement against PINY's own forces at each
RESPA level (fixtures made by tests/golden/make_golden.py, ``piny_ref respa``)
and the host-side set-up against the values PINY formed."""
import numpy as np
import pytest

from helpers import RESPA_NAMES, fixture_level, load_fixture, pair_hash, respa_from_fixture, rel_rms
from piny_b200 import respa as R


@pytest.mark.parametrize("name", RESPA_NAMES)
def test_respa_weights_match_piny(name):
    F = load_fixture(name)
    r = respa_from_fixture(F)
    for k in ("wght_ter", "wght_ter_res", "wght_tra_res"):
        assert r[k] == F[k], k


@pytest.mark.parametrize("name", RESPA_NAMES)
def test_respa_oracle_matches_piny(name, oracle):
    F = load_fixture(name)
    r = respa_from_fixture(F)
    xmod = F.get("xmod")
    pi, pj = oracle.verlist(F, F["pos"][0], xmod, F["hmat"], F["cutskin2"])
    assert pair_hash(pi, pj) == F["pairs_sha256"]
    for lv in range(4):
        f, ft = oracle.respa_force(F, r, fixture_level(F, lv), F["pos"], xmod, F["hmat"], pi, pj)
        assert rel_rms(f, F["ref_L%d_force_raw" % lv]) < 1e-13, lv
        if lv == 0 and "ref_L0_forcet_raw" in F:
            assert rel_rms(ft, F["ref_L0_forcet_raw"]) < 1e-13
    # the full level with every weight 1 is the plain evaluation, and so are
    # PINY's virial forces of the full level -- except with the separate
    # RESPA PME mesh, whose forces PINY adds to the virial forces too at the
    # full step (ewald3d_pme.c:563-585 runs for both meshes)
    plain, _ = oracle.energy_force(F, F["pos"], xmod, F["hmat"], pi, pj)
    one = dict(r, wght_ter=1.0, wght_ter_res=1.0, wght_tra_res=1.0)
    f, ft = oracle.respa_force(F, one, R.FULL_INTER | R.FULL_INTRA | R.RES_INTRA, F["pos"], xmod, F["hmat"], pi, pj)
    assert rel_rms(f, plain) < 1e-13
    assert rel_rms(ft, plain) < 1e-13
    if "ref_L0_forcet_raw" in F and not int(F.get("pme_res_on", 0)):
        assert rel_rms(plain, F["ref_L0_forcet_raw"]) < 1e-13


@pytest.mark.parametrize("name", ["respa_kspace_tip4pf_64_p4", "respa_pmegrid_tip4pf_64_p4"])
def test_ecor_res_table_matches_piny(name):
    """The exclusion correction's RESPA force table from piny_b200.system
    against PINY's ecor.cdv0_res: RESPA k cutoff equal to the full one (one
    PME grid) and smaller (PINY's separate RESPA grid)."""
    from piny_b200 import system
    F = load_fixture(name)
    t = system.ecor_res_table(int(F["ecor_nsplin"]), float(F["ecor_rmax"]), float(F["alp_ewd"]),
                              float(F["ecor_ecut"]), float(F["ecor_ecut_res"]))
    ref = F["ecor_cdv0_res"]
    # as for the plain table: Gauss-Legendre nodes computed here, PINY's
    # are tabulated (weights_nodes_128.h)
    assert np.abs(t - ref).max() <= 1e-10 * np.abs(ref).max()
    if name == "respa_pmegrid_tip4pf_64_p4":
        assert np.abs(ref - F["ecor_cdv0"]).max() > 1e-6 * np.abs(ref).max()


def test_respa_pme_mesh_matches_piny():
    """PINY's separate RESPA PME mesh (ewald_respa_pme_opt on): the host
    set-up's mesh, RESPA k sphere and B-spline weights against PINY's."""
    from piny_b200 import system
    F = load_fixture("respa_pmegrid_tip4pf_64_p4")
    m = system.pme_res_mesh(F["hmat"], int(F["kmax_res"]), int(F["kmax_pme_res"]), int(F["n_interp_res"]))
    assert list(m["ngrid_res"]) == list(F["ngrid_res"])
    for k in ("kastr_res", "kbstr_res", "kcstr_res"):
        assert np.array_equal(m[k], F[k]), k
    assert np.abs(m["bweight_res"] - F["bweight_tot_res"]).max() <= 1e-14 * np.abs(F["bweight_tot_res"]).max()


def test_respa_loop_levels():
    """int_NVT_pimd's nesting: the last call of a step is the full level,
    inner inter calls close each (tor, tra) sweep, the rest are innermost."""
    lv = R.loop_levels(2, 1, 2, 1, True)
    full = R.FULL_INTER | R.RES_INTER | R.FULL_INTRA | R.RES_INTRA
    inner = R.RES_INTER | R.FULL_INTRA | R.RES_INTRA
    assert lv == [R.RES_INTRA, inner, R.RES_INTRA, full]
    assert R.loop_levels(1, 1, 1, 3, False) == [0, 0, R.FULL_INTER | R.FULL_INTRA | R.RES_INTRA]
    assert R.loop_levels(1, 1, 2, 2, False) == [0, R.RES_INTRA, 0, R.FULL_INTER | R.FULL_INTRA | R.RES_INTRA]


def test_oracle_respa_step_reduces_to_plain(oracle):
    """The oracle's RESPA step with every count 1 and unit weights is its
    plain NVT step."""
    from oracle import oracle as O
    from piny_b200 import pimd, system, water
    spec = water.BoxSpec(water.TIP4P_F, 27, water.density_box_edge(27), 4, 298.0, 21, grid=16, order=8,
                         cutoff=4.5)
    pos = water.build_positions(spec) / water.BOHR
    S = system.build_system(spec, pos)
    natm = int(S["natm"])
    ghost = np.zeros(natm, bool)
    ghost[np.asarray(S["ghost_atom"])] = True
    mass = np.tile(np.asarray(spec.model.masses, np.float64), spec.nmol) * 1822.888486
    setup = pimd.nvt_setup(mass, ghost, 4, 2, spec.temperature, 20.0, 800.0, len_nhc=3)
    rs = R.respa_setup(1, 1, 1, 1, True, False, np.asarray(S["cutoff"]), 1.0, np.asarray(S["bond_eq"]))
    rng = np.random.default_rng(2)
    v = rng.normal(size=(4, natm, 3)) * 1e-4
    v[:, ghost, :] = 0.0
    c, b = setup["class_nhc"], setup["bead_nhc"]
    st = {"cx": rng.normal(0, 0.05, (c["len_nhc"], c["num_nhc"])), "cv": rng.normal(0, 1e-4, (c["len_nhc"], c["num_nhc"])),
          "bx": rng.normal(0, 0.05, (3, b["len_nhc"], b["num_nhc"])), "bv": rng.normal(0, 1e-4, (3, b["len_nhc"], b["num_nhc"]))}
    st2 = {k: a.copy() for k, a in st.items()}
    x0 = O.ghost_positions(S, pos)
    u0 = oracle.pimd_transform(x0, 2, 0)
    pi, pj = oracle.verlist(S, x0[0], u0[0], S["hmat"], S["cutskin2"])
    x, f = O.pimd_forces(oracle, S, setup, pos, pi, pj)[:2]
    a = O.pimd_step(oracle, S, setup, x, v, f, st, pi, pj)
    b2 = O.pimd_step_respa(oracle, S, setup, rs, x, v, f, st2, pi, pj)
    for k in range(3):
        assert np.abs(a[k] - b2[k]).max() <= 1e-12 * np.abs(a[k]).max(), k
    assert abs(a[3]["akvirx"] - b2[3]["akvirx"]) <= 1e-12 * abs(a[3]["akvirx"])
    for k in st:
        assert np.abs(st[k] - st2[k]).max() <= 1e-12 * max(np.abs(st[k]).max(), 1e-30), k
