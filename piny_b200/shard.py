"""Splitting the work of the force path over ranks (one process per GPU).

Beads and boxes are independent units: no data-path exchange is needed.
A box's P beads can be split into contiguous ranges, one per rank; every
rank builds the same list (from bead 1 of the whole box and the shared
mode-1 positions, so the images are PINY's) and evaluates its own range.
The only exchange is one all-reduce of the energy components and the
pressure tensor, a few hundred bytes per step:
  energies are bead averages, so a rank's averages weigh P_rank / P;
  pvten is a bead sum (PINY's pvten_tot), so the ranks' tensors add.
Independent boxes (replicas) need no exchange at all.
"""
from __future__ import annotations

import numpy as np

ENERGY_KEYS = ("vreal", "vvdw", "vcoul", "vrecip", "vself", "vbgr", "vecor", "vlong", "vbond", "vbend", "vintert",
               "vintrat")


def bead_range(nbeads: int, world: int, rank: int):
    """Contiguous bead range [b0, b1) of `rank`: equal power-of-two slices
    (the device path takes 1, 2, 4, ..., 64 beads per context)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad world/rank")
    if nbeads % world:
        raise ValueError("%d beads do not split evenly over %d ranks" % (nbeads, world))
    per = nbeads // world
    if per & (per - 1):
        raise ValueError("beads per rank must be a power of two, got %d" % per)
    return rank * per, (rank + 1) * per


def item_range(n: int, world: int, rank: int):
    """Contiguous share [i0, i1) of n independent items (boxes) for `rank`;
    the first n % world ranks take one more."""
    base, extra = divmod(n, world)
    i0 = rank * base + min(rank, extra)
    return i0, i0 + base + (1 if rank < extra else 0)


def combine_bead_shards(e: dict, nbeads_local: int, nbeads_total: int, group=None) -> dict:
    """The whole box's energies from this rank's (over its own beads), by one
    FP64 all-reduce: energies weighted by P_rank / P, pvten summed."""
    import torch
    import torch.distributed as dist
    w = float(nbeads_local) / float(nbeads_total)
    vec = torch.tensor([e[k] * w for k in ENERGY_KEYS] + list(np.asarray(e["pvten"], np.float64)),
                       dtype=torch.float64)
    if dist.is_available() and dist.is_initialized():
        if dist.get_backend(group) == "nccl":
            vec = vec.cuda()
        dist.all_reduce(vec, op=dist.ReduceOp.SUM, group=group)
        vec = vec.cpu()
    out = {k: float(vec[i]) for i, k in enumerate(ENERGY_KEYS)}
    out["pvten"] = vec[len(ENERGY_KEYS):].numpy().copy()
    return out
