"""Graph replay of the single-box entry points.

A call with the same pointers, cell, flags and stream as the one before is
a replay of one captured CUDA graph; the inputs behind the pointers may
change between calls.  Every call (plain, captured, replayed) must give the
oracle's forces and energies for the positions it was given: FP64 relative
RMS 1e-12.
"""
import numpy as np
import pytest

from helpers import load_fixture, rel_rms

pytestmark = pytest.mark.gpu


def test_replayed_evaluations_follow_the_inputs(oracle):
    import torch

    from piny_b200.lib import DeviceBox

    F = load_fixture("tip4pf_64_p4")
    P = int(F["nbeads"])
    xmod = F["xmod"]
    box = DeviceBox(F, P, "fp64")
    box.build_list(F["pos"][0], xmod, F["hmat"], F["cutskin2"])
    pi, pj = box.get_list()
    rng = np.random.default_rng(3)
    inputs = [F["pos"] + rng.normal(scale=0.01, size=F["pos"].shape) for _ in range(4)]
    dev = torch.device("cuda:0")
    d = torch.from_numpy(np.ascontiguousarray(inputs[0])).to(dev)
    dx = torch.from_numpy(np.ascontiguousarray(xmod)).to(dev)
    f = torch.zeros_like(d)
    for k in [0, 0, 1, 2, 3, 1]:  # plain, captured, then replays with new contents
        d.copy_(torch.from_numpy(inputs[k]))
        e = box.energy_force_device(d.data_ptr(), dx.data_ptr(), F["hmat"], f.data_ptr())
        fref, eref = oracle.energy_force(F, inputs[k], xmod, F["hmat"], pi, pj)
        assert rel_rms(f.cpu().numpy(), fref) < 1e-12, k
        assert abs(e["vintert"] - eref["vintert"]) <= 1e-11 * max(1.0, abs(eref["vintert"])), k
        assert abs(e["vintrat"] - eref["vintrat"]) <= 1e-11 * max(1.0, abs(eref["vintrat"])), k
        assert box.last_timing()[0] > 0.0
    # the host-buffer entry replays its own graph the same way
    for k in [2, 2, 0, 3]:
        fh, eh = box.energy_force(inputs[k], xmod, F["hmat"])
        fref, eref = oracle.energy_force(F, inputs[k], xmod, F["hmat"], pi, pj)
        assert rel_rms(fh, fref) < 1e-12, k
        assert abs(eh["vintert"] - eref["vintert"]) <= 1e-11 * max(1.0, abs(eref["vintert"])), k
    # a new cell is a new graph
    h2 = np.asarray(F["hmat"]) * 1.002
    for k in [1, 1, 1]:
        fh, eh = box.energy_force(inputs[k], xmod, h2)
        fref, eref = oracle.energy_force(F, inputs[k], xmod, h2, pi, pj)
        assert rel_rms(fh, fref) < 1e-12
    box.close()
