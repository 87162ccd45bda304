"""The oracle's row-range list (orc_verlist_rows) is the full list's rows."""
import numpy as np

from helpers import load_fixture, pair_hash


def test_rows_are_the_full_lists_rows(oracle):
    F = load_fixture("tip4pf_64_p4")
    pos = np.ascontiguousarray(F["pos"], np.float64)
    xm = pos.mean(axis=0)
    pi, pj = oracle.verlist(F, pos[0], xm, F["hmat"], F["cutskin2"])
    for lo, hi in ((0, 40), (37, 150), (200, 256), (0, 256)):
        ri, rj = oracle.verlist_rows(F, pos[0], xm, F["hmat"], F["cutskin2"], lo, hi)
        sel = (pi >= lo) & (pi < hi)
        assert pair_hash(ri, rj) == pair_hash(pi[sel], pj[sel])
