"""The PINY input reader behind PINYEmpirical: a directory written in PINY's
input language reads back to the same box, and the host set-up built from
it is the one built from the original specification (bit for bit)."""
import numpy as np
import pytest

from piny_b200 import empirical, system, water


@pytest.mark.parametrize("spec", [
    water.BoxSpec(water.TIP4P_F, 64, 12.416, 1, 298.0, 103, cutoff=6.0, grid=16, order=8, kmax=6),
    water.BoxSpec(water.SPC_FW, 64, 12.416, 1, 300.0, 101, cutoff=6.0, grid=16, order=6, kmax=6),
])
def test_input_directory_reads_back(spec, tmp_path):
    pos = water.build_positions(spec)
    water.write_piny_input(str(tmp_path), spec, pos)
    spec2, pos2 = empirical.read_water_input(str(tmp_path), "water.input")
    assert np.array_equal(pos2, pos / water.BOHR)
    assert spec2.nmol == spec.nmol and spec2.L == spec.L and spec2.nbeads == 1
    assert spec2.model.sites == spec.model.sites and spec2.model.charges == spec.model.charges
    S1 = system.build_system(spec, pos / water.BOHR)
    S2 = system.build_system(spec2, pos2)
    for k in ("atm_typ", "inter_map", "excl_off", "excl_j", "kastr", "kbstr", "kcstr", "bond_j1", "bend_j1"):
        assert np.array_equal(np.asarray(S1[k]), np.asarray(S2[k])), k
    for k in ("charge", "cutoff", "cutskin2", "cv0", "cdv0", "cv0_c", "cdv0_c", "bweight", "bond_c", "bond_eq",
              "bend_c", "bend_s", "ecor_cv0", "hmat"):
        a, b = np.asarray(S1[k], np.float64), np.asarray(S2[k], np.float64)
        assert np.allclose(a, b, rtol=1e-13, atol=0), k
    for k in ("alp_ewd", "clong", "nktot", "ngrid_a", "n_interp", "nghost"):
        assert S1.get(k) == pytest.approx(S2.get(k), rel=1e-13), k


def test_path_integral_input_is_refused(tmp_path):
    pytest.importorskip("torch")
    spec = water.BoxSpec(water.TIP4P_F, 64, 12.416, 2, 298.0, 3, cutoff=6.0, grid=16, order=8, kmax=6)
    water.write_piny_input(str(tmp_path), spec, water.build_positions(spec))
    sp, pos = empirical.read_water_input(str(tmp_path), "water.input")
    assert sp.nbeads == 2 and pos.shape[0] == 2
