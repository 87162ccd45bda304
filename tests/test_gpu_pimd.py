"""Device ring-polymer transforms (pinyb200_pimd_transform) against the
oracle and PINY's own outputs.

Staging: bit-identical to the oracle and to PINY (the oracle is, too).
Normal modes: within 4e-15 of the row scale of the oracle and of PINY
(direct sums against PINY's FFT; both FP64).  At a full box (4096 water
molecules, 12288 atoms, 32 and 64 beads) the device is checked against the
oracle the same way, and through the round trip and transpose identities."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pimd_transforms.npz")
NM_TOL = 4e-15


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, np.float64)).to("cuda:0")


def _run(x, kind, what):
    import torch

    from piny_b200 import lib
    d = _dev(x)
    P, natm = x.shape[0], x.shape[1]
    lib.pimd_transform(d.data_ptr(), natm, P, kind, what, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return d.cpu().numpy()


def _close(a, b, kind):
    if kind == 1:
        return np.array_equal(a, b)
    return np.abs(a - b).max() <= NM_TOL * max(1.0, np.abs(b).max())


@pytest.mark.parametrize("kind,P", [(1, 2), (1, 4), (1, 8), (1, 32), (1, 64), (2, 2), (2, 4), (2, 8), (2, 16),
                                    (2, 32), (2, 64)])
def test_device_matches_piny_fixture(kind, P):
    g = np.load(GOLD)
    t = "k%d_p%d_" % (kind, P)
    assert _close(_run(g[t + "x"], kind, 0), g[t + "modes"], kind)
    assert _close(_run(g[t + "modes"], kind, 1), g[t + "back"], kind)
    assert _close(_run(g[t + "f"], kind, 2), g[t + "fmodes"], kind)


@pytest.mark.parametrize("kind", [1, 2])
@pytest.mark.parametrize("P", [32, 64])
def test_device_full_box(oracle, kind, P):
    rng = np.random.default_rng(100 * kind + P)
    natm = 12288
    x = rng.uniform(0, 46.9, size=(1, natm, 3)) + rng.normal(0, 0.3, size=(P, natm, 3))
    f = rng.normal(0, 0.05, size=(P, natm, 3))
    u = _run(x, kind, 0)
    assert _close(u, oracle.pimd_transform(x, kind, 0), kind)
    back = _run(u, kind, 1)
    assert _close(back, oracle.pimd_transform(u, kind, 1), kind)
    assert np.abs(back - x).max() <= 1e-13 * np.abs(x).max()
    fu = _run(f, kind, 2)
    assert _close(fu, oracle.pimd_transform(f, kind, 2), kind)
    du = rng.normal(size=x.shape)
    lhs = np.einsum("bid,bid->id", fu, du)
    rhs = np.einsum("bid,bid->id", f, _run(du, kind, 1))
    assert np.abs(lhs - rhs).max() <= 1e-12 * np.abs(rhs).max()


def test_ragged_atom_counts(oracle):
    """Atom counts that leave the last block partly empty."""
    rng = np.random.default_rng(5)
    for natm in (1, 43, 129):
        for kind in (1, 2):
            x = rng.normal(size=(8, natm, 3))
            for what in (0, 1, 2):
                assert _close(_run(x, kind, what), oracle.pimd_transform(x, kind, what), kind)


def test_arguments():
    from piny_b200 import lib
    from piny_b200.lib import PinyError
    d = _dev(np.arange(12.0).reshape(1, 4, 3))
    lib.pimd_transform(d.data_ptr(), 4, 1, lib.NORMAL_MODES, lib.TO_MODES)  # one bead: no-op
    assert np.array_equal(d.cpu().numpy(), np.arange(12.0).reshape(1, 4, 3))
    with pytest.raises(PinyError, match="ERR_UNSUPPORTED"):
        lib.pimd_transform(d.data_ptr(), 1, 3, lib.STAGING, lib.TO_MODES)
    with pytest.raises(PinyError, match="ERR_ARG"):
        lib.pimd_transform(d.data_ptr(), 4, 1, 7, lib.TO_MODES)
    with pytest.raises(PinyError, match="ERR_ARG"):
        lib.pimd_transform(d.data_ptr(), 0, 2, lib.STAGING, lib.TO_MODES)
