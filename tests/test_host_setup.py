"""The product's numpy host set-up against PINY's set-up products."""
import numpy as np
import pytest

from helpers import GOLDEN_NAMES, load_fixture, spec_from_fixture
from piny_b200 import system

EXACT_INT = ["atm_typ", "inter_map", "excl_off", "excl_j", "kastr", "kbstr", "kcstr", "bond_j1", "bond_j2",
             "bend_j1", "bend_j2", "bend_j3", "ghost_atom", "ghost_comp"]
CLOSE = {"charge": 0, "cutoff": 1e-15, "rmin_spl": 1e-15, "dr_spl": 1e-15, "dri_spl": 1e-15, "cv0": 1e-14,
         "cdv0": 1e-14, "cv0_c": 1e-14, "cdv0_c": 1e-14, "skin": 1e-15, "clong": 1e-13, "alp_ewd": 1e-15,
         "self_erf": 1e-15, "bweight": 1e-14, "ecor_rmax": 1e-14, "ecor_dr": 1e-14, "bond_eq": 1e-15,
         "bond_c": 1e-14, "bond_dc": 1e-14, "bend_c": 1e-14, "bend_s": 1e-14, "bend_dc": 1e-14,
         "bend_ds": 1e-14, "ghost_coef": 0, "spread": 1e-13, "cutskin2": 1e-14, "hmat": 1e-15}


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_host_setup_matches_piny(name):
    F = load_fixture(name)
    S = system.build_system(spec_from_fixture(F), F["pos"])
    for k in EXACT_INT:
        if k in F:
            assert np.array_equal(np.asarray(S[k]), np.asarray(F[k])), k
    for k, tol in CLOSE.items():
        if k not in F:
            continue
        a, b = np.asarray(S[k], np.float64), np.asarray(F[k], np.float64)
        scale = np.maximum(np.abs(b), 1e-300)
        assert np.all(np.abs(a - b) <= tol * scale + 1e-300), k
    for k in ("nktot", "ngrid_a", "ngrid_b", "ngrid_c", "n_interp", "necor", "nbond", "nbend", "nghost",
              "ninter_unique", "nsplin"):
        assert int(S[k]) == int(F[k]), k
    # same Ewald-correction pair set (PINY's order follows its exclusion walk)
    a = set(zip(S["ecor_j1"].tolist(), S["ecor_j2"].tolist()))
    b = set(zip(F["ecor_j1"].tolist(), F["ecor_j2"].tolist()))
    assert a == b
    # the correction table agrees where the pairs live (r > 1 Bohr)
    r = F["ecor_rmin"] + F["ecor_dr"] * (np.arange(F["ecor_nsplin"]) - 2.0)
    m = r > 1.0
    assert np.max(np.abs(S["ecor_cv0"][m] - F["ecor_cv0"][m])) < 1e-13 * np.abs(F["ecor_cv0"]).max()
    assert np.max(np.abs(S["ecor_cdv0"][m] - F["ecor_cdv0"][m])) < 1e-12 * np.abs(F["ecor_cdv0"]).max()
