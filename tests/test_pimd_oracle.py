"""Ring-polymer transforms of the oracle (orc_pimd_transform) against PINY's
own (tests/golden/pimd_transforms.npz, made by ``piny_ref pimd`` from PINY's
path_integral_init and convert_pimd_{mode,pos,force}_{stag,cent}), and the
identities the transforms obey at any size:
  * modes -> positions inverts positions -> modes;
  * mode forces are the transpose of the modes -> positions map applied to
    the bead forces (F_u . du = f . x(du) for every du), which is what makes
    them forces on the modes;
  * mode 1 of the normal modes is the centroid, and its mode force the total.
Staging must be bit-identical to PINY; normal modes agree to rounding
(PINY's FFT against the oracle's direct sums): 4e-15 of the row scale."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pimd_transforms.npz")
CASES = [(1, 2), (1, 4), (1, 6), (1, 8), (1, 32), (1, 64), (2, 2), (2, 4), (2, 8), (2, 16), (2, 32), (2, 64)]
NM_TOL = 4e-15


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _close(a, b, kind):
    if kind == 1:
        return np.array_equal(a, b)
    return np.abs(a - b).max() <= NM_TOL * max(1.0, np.abs(b).max())


@pytest.mark.parametrize("kind,P", CASES)
def test_oracle_transforms_match_piny(gold, oracle, kind, P):
    t = "k%d_p%d_" % (kind, P)
    x, f = gold[t + "x"], gold[t + "f"]
    assert _close(oracle.pimd_transform(x, kind, 0), gold[t + "modes"], kind)
    assert _close(oracle.pimd_transform(gold[t + "modes"], kind, 1), gold[t + "back"], kind)
    assert _close(oracle.pimd_transform(f, kind, 2), gold[t + "fmodes"], kind)


@pytest.mark.parametrize("kind,P", [(1, 5), (1, 32), (2, 8), (2, 64)])
def test_transform_identities(oracle, kind, P):
    rng = np.random.default_rng(P + 10 * kind)
    natm = 40
    x = rng.uniform(0, 30, size=(1, natm, 3)) + rng.normal(0, 0.4, size=(P, natm, 3))
    u = oracle.pimd_transform(x, kind, 0)
    assert np.abs(oracle.pimd_transform(u, kind, 1) - x).max() <= 1e-13 * np.abs(x).max()
    # mode forces = J^T f with J the (linear) modes -> positions map
    f = rng.normal(size=(P, natm, 3))
    du = rng.normal(size=(P, natm, 3))
    fu = oracle.pimd_transform(f, kind, 2)
    lhs = np.einsum("bid,bid->id", fu, du)
    rhs = np.einsum("bid,bid->id", f, oracle.pimd_transform(du, kind, 1))
    assert np.abs(lhs - rhs).max() <= 1e-12 * np.abs(rhs).max()
    if kind == 2:
        assert np.abs(u[0] - x.mean(axis=0)).max() <= 1e-13 * np.abs(x).max()
        assert np.abs(fu[0] - f.sum(axis=0)).max() <= 1e-13 * np.abs(f).sum(axis=0).max()
    else:
        assert np.array_equal(u[0], x[0])  # staging keeps bead 1


def test_normal_modes_agree_with_numpy_fft(oracle):
    rng = np.random.default_rng(3)
    P, natm = 16, 7
    x = rng.normal(size=(P, natm, 3))
    u = oracle.pimd_transform(x, 2, 0)
    X = np.fft.ifft(x, axis=0)  # (1/P) sum_j x_j e^{+2 pi i jk/P}
    want = np.empty_like(x)
    want[0] = X[0].real
    want[P - 1] = X[P // 2].real
    for m in range(1, P // 2):
        want[2 * m - 1] = X[m].real
        want[2 * m] = X[m].imag
    assert np.abs(u - want).max() <= 1e-14 * np.abs(x).max()


def test_bad_arguments(oracle):
    with pytest.raises(ValueError):
        oracle.pimd_transform(np.zeros((6, 2, 3)), 2, 0)  # normal modes need 2^n beads
    with pytest.raises(ValueError):
        oracle.pimd_transform(np.zeros((4, 2, 3)), 3, 0)
    x = np.arange(6.0).reshape(1, 2, 3)
    assert np.array_equal(oracle.pimd_transform(x, 1, 0), x)  # one bead: untouched


# -- chains, springs, centroid virial, set-up (pimd_md.npz) ------------------

MD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pimd_md.npz")


@pytest.fixture(scope="module")
def md():
    return np.load(MD)


def _chains(g, t):
    return {"num_nhc": int(g[t + "num"]), "len_nhc": int(g[t + "len"]), "nres_nhc": int(g[t + "nres"]),
            "wdti": g[t + "wdti"], "inhc": g[t + "inhc"], "mass_nhc": g[t + "mass_nhc"], "gkt": g[t + "gkt"]}


@pytest.mark.parametrize("case", [0, 1, 2])
def test_oracle_chains_match_piny(md, oracle, case):
    from oracle.oracle import nhc_apply
    t = "nhc%d_" % case
    v, x, vn = nhc_apply(oracle, md[t + "v"], md[t + "mass"], _chains(md, t), md[t + "x_nhc"], md[t + "v_nhc"])
    assert np.array_equal(v, md[t + "ref_v"])
    assert np.array_equal(x, md[t + "ref_x_nhc"])
    assert np.array_equal(vn, md[t + "ref_v_nhc"])


@pytest.mark.parametrize("case", [0, 1, 2])
def test_yoshida_weights_match_piny(md, case):
    from piny_b200.pimd import yoshida_weights
    t = "nhc%d_" % case
    assert np.array_equal(yoshida_weights(int(md[t + "nyosh"]), float(md[t + "dti"])), md[t + "wdti"])


@pytest.mark.parametrize("P", [4, 8])
def test_oracle_springs_and_virial_match_piny(md, oracle, P):
    from oracle.oracle import pimd_force_post, pimd_springs
    from piny_b200.water import BOLTZ
    t = "spr_p%d_" % P
    fm, ake, pvm = pimd_springs(oracle, md[t + "u"], md[t + "prekf"], md[t + "veig"], float(md[t + "wght"]))
    assert np.array_equal(fm, md[t + "ref_fm"])
    assert ake == md[t + "ref_kin_harm"]
    assert np.array_equal(pvm, md[t + "ref_pvten_mode_tot"])
    # PINY's routine takes forces and tensors already divided by P; P is a
    # power of two, so scaling the inputs by P first is exact
    natm = md[t + "u"].shape[1]
    _, akv, pv, pvt = pimd_force_post(oracle, 1, md[t + "f"] * P, md[t + "x"], md[t + "xmod"], np.zeros_like(fm), natm,
                                      BOLTZ / float(md[t + "T"]), md[t + "pvten"] * P, md[t + "pvten_tot"] * P)
    assert np.array_equal(pv, md[t + "ref_pvten"])
    assert np.array_equal(pvt, md[t + "ref_pvten_tot"])
    assert akv == md[t + "ref_akvirx"]


@pytest.mark.parametrize("kind,P", CASES)
def test_path_integral_setup_matches_piny(gold, kind, P):
    from piny_b200.pimd import path_integral_setup
    t = "k%d_p%d_" % (kind, P)
    mass = gold["mass"]
    s = path_integral_setup(mass, P, kind, 300.0)
    assert np.allclose(s["path_eig"], gold[t + "path_eig"], rtol=1e-15, atol=0)
    assert np.allclose(s["bead_mass"], gold[t + "bead_mass"], rtol=1e-15, atol=0)
    assert np.array_equal(s["prekf"], gold[t + "prekf"])
