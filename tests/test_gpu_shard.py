"""Bead sharding over 2 ranks on the device library: each rank (a process of
its own, both on cuda:0 here; on a multi-GPU node one GPU each) builds the
whole box's list from bead 1 and the shared mode-1 positions, evaluates its
own bead range with a DeviceBox, and one gloo all-reduce of the energies
(shard.combine_bead_shards) reproduces the one-process device result:
FP64 energies and pressure tensor to 1e-12 relative, forces of each range
to 1e-12 of the largest force.  The ranks' kernels never wait on each
other; the only exchange is the host-side all-reduce."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from piny_b200 import shard

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from helpers import load_fixture
    from piny_b200.lib import DeviceBox
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        F = load_fixture("tip4pf_64_p4")
        P = int(F["nbeads"])
        b0, b1 = shard.bead_range(P, world, rank)
        box = DeviceBox(F, b1 - b0, "fp64")
        box.build_list(F["pos"][0], F["xmod"], F["hmat"], F["cutskin2"])
        f, e = box.energy_force(F["pos"][b0:b1], F["xmod"], F["hmat"])
        box.close()
        tot = shard.combine_bead_shards(e, b1 - b0, P)
        out[rank] = (tot, f, b0, b1)
    finally:
        dist.destroy_process_group()


def test_two_rank_device_bead_shards_match_one_process():
    from helpers import load_fixture
    from piny_b200.lib import DeviceBox
    F = load_fixture("tip4pf_64_p4")
    box = DeviceBox(F, int(F["nbeads"]), "fp64")
    box.build_list(F["pos"][0], F["xmod"], F["hmat"], F["cutskin2"])
    f_all, e_all = box.energy_force(F["pos"], F["xmod"], F["hmat"])
    box.close()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    for r in range(2):
        tot, f, b0, b1 = out[r]
        for k in shard.ENERGY_KEYS:
            assert abs(tot[k] - e_all[k]) <= 1e-12 * max(1.0, abs(e_all[k])), k
        assert np.abs(tot["pvten"] - e_all["pvten"]).max() <= 1e-12 * np.abs(e_all["pvten"]).max()
        assert np.abs(f - f_all[b0:b1]).max() <= 1e-12 * np.abs(f_all).max()
