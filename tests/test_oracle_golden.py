"""The oracle restatement against PINY's own outputs (golden fixtures made by
tests/golden/make_golden.py from PINY built from its sources)."""
import numpy as np
import pytest

from helpers import GOLDEN_NAMES, load_fixture, pair_hash, rel_rms

ENERGY_KEYS = [("vintert", "vintert"), ("vintrat", "vintrat"), ("vvdw", "vvdw"), ("vcoul", "vcoul"),
               ("vlong", "vlong"), ("vbond", "vbondt"), ("vbend", "vbendt")]


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_oracle_matches_piny(name, oracle):
    F = load_fixture(name)
    xmod = F.get("xmod")
    pi, pj = oracle.verlist(F, F["pos"][0], xmod, F["hmat"], F["cutskin2"])
    # bit-exact pair set
    assert len(pi) == F["npairs"]
    assert pair_hash(pi, pj) == F["pairs_sha256"]
    force, e = oracle.energy_force(F, F["pos"], xmod, F["hmat"], pi, pj, distribute_ghosts=False)
    assert rel_rms(force, F["ref_force_raw"]) < 1e-13
    force2, _ = oracle.energy_force(F, F["pos"], xmod, F["hmat"], pi, pj, distribute_ghosts=True)
    assert rel_rms(force2, F["ref_force"]) < 1e-13
    for k, kr in ENERGY_KEYS:
        assert abs(e[k] - F["ref_" + kr]) <= 1e-12 * max(1.0, abs(F["ref_" + kr])), k
    vrec = e["vrecip"] + e["vself"] + e["vbgr"] + e["vecor"]
    assert abs(vrec - F["ref_vrecip"]) <= 1e-12 * max(1.0, abs(F["ref_vrecip"]))
    assert np.abs(e["pvten"] - F["ref_pvten_tot"]).max() <= 1e-12 * np.abs(F["ref_pvten_tot"]).max()


@pytest.mark.parametrize("name", ["spcfw_64_p1", "tip4pf_64_p4"])
def test_oracle_pair_list_order_free(name, oracle):
    """The stored pair list (PINY order) and the oracle's agree pair by pair."""
    F = load_fixture(name)
    pi, pj = oracle.verlist(F, F["pos"][0], F.get("xmod"), F["hmat"], F["cutskin2"])
    a = set(zip(pi.tolist(), pj.tolist()))
    b = set(map(tuple, F["pairs"].tolist()))
    assert a == b


def test_oracle_setup_tables(oracle):
    """Oracle set-up restatements reproduce PINY's tables."""
    F = load_fixture("tip4pf_64_p4")
    nsplin = F["nsplin"]
    u_lj = int(F["inter_map"][0])
    from piny_b200.water import BOHR, BOLTZ, KB_KCAL, TIP4P_F
    eps = (TIP4P_F.lj_eps_kcal / KB_KCAL) / BOLTZ
    sig = TIP4P_F.lj_sigma / BOHR
    rmin, rmax = F["rmin_spl"][u_lj], F["cutoff"][0]
    v, dv, dr, dri = oracle.spline_table(nsplin, rmin, rmax, 2, sig, eps, 0.0, 1.0 / BOHR, 2)
    ref_v = F["cv0"][u_lj * nsplin:(u_lj + 1) * nsplin]
    ref_dv = F["cdv0"][u_lj * nsplin:(u_lj + 1) * nsplin]
    assert np.max(np.abs(v - ref_v) / np.maximum(np.abs(ref_v), 1e-300)) < 1e-14
    assert np.max(np.abs(dv - ref_dv) / np.maximum(np.abs(ref_dv), 1e-300)) < 1e-14
    vc, dvc, _, _ = oracle.spline_table(nsplin, rmin, rmax, 1, 1.0, 0.0, F["alp_ewd"], 1.0 / BOHR, 2)
    assert np.max(np.abs(vc - F["cv0_c"][:nsplin])) < 1e-14 * np.abs(F["cv0_c"]).max()
    ecut, kmaxv, ka, kb, kc = oracle.kvectors(int(F["spec_kmax"]), F["hmat"])
    assert len(ka) == F["nktot"]
    assert np.array_equal(ka, F["kastr"]) and np.array_equal(kb, F["kbstr"]) and np.array_equal(kc, F["kcstr"])
    ng = oracle.pme_grid(ecut, F["hmat"], kmaxv, int(F["spec_kmax_pme"]))
    assert list(ng) == [F["ngrid_a"], F["ngrid_b"], F["ngrid_c"]]
    bw = oracle.bweight(ka, kb, kc, ng, F["n_interp"])
    assert np.max(np.abs(bw - F["bweight"]) / F["bweight"]) < 1e-14
    cv0, cdv0, edr, edri, self_erf = oracle.ecor_table(F["ecor_nsplin"], F["ecor_rmax"], F["alp_ewd"],
                                                       F["ecor_ecut"])
    assert abs(edr - F["ecor_dr"]) <= 1e-15 * F["ecor_dr"]
    assert np.max(np.abs(cv0 - F["ecor_cv0"])) < 1e-12 * np.abs(F["ecor_cv0"]).max()
    assert np.max(np.abs(cdv0 - F["ecor_cdv0"])) < 1e-10 * np.abs(F["ecor_cdv0"]).max()
    assert abs(self_erf - F["self_erf"]) < 1e-15
    c, s, dc, ds = oracle.bend_harm((TIP4P_F.bend_k_kcal / KB_KCAL) / BOLTZ, TIP4P_F.bend_theta0 * (np.pi / 180.0))
    assert np.allclose(c, F["bend_c"], rtol=1e-14, atol=0) and np.allclose(s, F["bend_s"], rtol=1e-14, atol=0)
    c6 = np.zeros(6)
    c6[0] = 4.0 * eps * sig ** 6
    cl = oracle.clong(F["atm_typ"], F["ntyp"], c6, F["cutoff"], 1.0 / BOHR, 1)
    assert abs(cl - F["clong"]) < 1e-12 * abs(F["clong"])


def test_oracle_list_check_matches_numpy(oracle):
    """The rebuild-test restatement against a direct numpy statement of
    check_ver_list / get_pimd_spread / get_cut_skin."""
    rng = np.random.default_rng(3)
    for P in (1, 4):
        x0 = rng.normal(size=(50, 3)) * 10
        pos = x0[None] + rng.normal(scale=0.3, size=(P, 50, 3))
        cutoff = np.array([17.0, 16.5, 15.0])
        for skin, spread_ref in ((1.89, 0.0), (0.5, 0.2), (3.0, 5.0)):
            f, rmax, sp, cs = oracle.check_list(pos, x0, skin, spread_ref, cutoff)
            r = np.sqrt(((pos[0] - x0) ** 2).sum(1).max())
            s = np.sqrt(((pos[1:] - pos[0][None]) ** 2).sum(2).max()) if P > 1 else 0.0
            assert rmax == pytest.approx(r, rel=1e-15) and sp == pytest.approx(s, rel=1e-15)
            assert f == (r > skin / 2 + (max(0.0, s - spread_ref) if P > 1 else 0.0))
            assert np.allclose(cs, (cutoff + skin + s) ** 2, rtol=1e-15)
