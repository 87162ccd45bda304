"""Bead sharding over 2 ranks (gloo, CPU): each rank evaluates its own bead
range with the oracle, using the whole box's list and mode-1 positions, and
one all-reduce of the energies reproduces the single-process result."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from piny_b200 import shard


def test_ranges():
    assert shard.bead_range(32, 2, 1) == (16, 32)
    assert shard.bead_range(32, 4, 0) == (0, 8)
    with pytest.raises(ValueError):
        shard.bead_range(32, 3, 0)
    with pytest.raises(ValueError):
        shard.bead_range(24, 2, 0)
    spans = [shard.item_range(10, 4, r) for r in range(4)]
    assert spans == [(0, 3), (3, 6), (6, 8), (8, 10)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from helpers import load_fixture
    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        O = Oracle()
        F = load_fixture("tip4pf_64_p4")
        P = int(F["nbeads"])
        xmod = F["xmod"]
        pi, pj = O.verlist(F, F["pos"][0], xmod, F["hmat"], F["cutskin2"])
        b0, b1 = shard.bead_range(P, world, rank)
        f, e = O.energy_force(F, F["pos"][b0:b1], xmod, F["hmat"], pi, pj)
        tot = shard.combine_bead_shards(e, b1 - b0, P)
        out[rank] = (tot, f, b0, b1)
    finally:
        dist.destroy_process_group()


def test_two_rank_bead_shards_match_one_process(oracle):
    from helpers import load_fixture
    F = load_fixture("tip4pf_64_p4")
    xmod = F["xmod"]
    pi, pj = oracle.verlist(F, F["pos"][0], xmod, F["hmat"], F["cutskin2"])
    f_all, e_all = oracle.energy_force(F, F["pos"], xmod, F["hmat"], pi, pj)
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        tot, f, b0, b1 = out[r]
        for k in shard.ENERGY_KEYS:
            assert abs(tot[k] - e_all[k]) <= 1e-12 * max(1.0, abs(e_all[k])), k
        assert np.abs(tot["pvten"] - e_all["pvten"]).max() <= 1e-12 * np.abs(e_all["pvten"]).max()
        assert np.abs(f - f_all[b0:b1]).max() <= 1e-12 * np.abs(f_all).max()
