"""Batched boxes (one CUDA graph per call) and launch shapes: every path
gives the forces and energies of the one-box path.

Tolerances: FP64 force relative RMS 1e-12 (the kernels are the same; only
atomic summation order differs), MIXED 1e-5 against the FP64 one-box result.
"""
import numpy as np
import pytest

from helpers import rel_rms

pytestmark = pytest.mark.gpu


def _boxes(nbox=4, seed=77):
    from piny_b200 import system, water
    specs = water.c4_specs(nbox=nbox, seed=seed, nmin=64, nmax=300)
    out = []
    for sp in specs:
        pos = water.build_positions(sp) / water.BOHR
        S = system.build_system(sp, pos)
        out.append((sp, pos, S))
    return out


def _single(S, pos, P, prec, choice=None):
    import torch

    from piny_b200.lib import DeviceBox
    box = DeviceBox(S, P, prec)
    xmod = pos.mean(axis=0) if P > 1 else None
    box.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
    if choice is not None:
        box.set_tuning(choice)
    d = torch.from_numpy(pos).to("cuda:0")
    dx = torch.from_numpy(xmod).to("cuda:0") if xmod is not None else None
    f = torch.empty_like(d)
    e = box.energy_force_device(d.data_ptr(), None if dx is None else dx.data_ptr(), S["hmat"], f.data_ptr())
    return box, f.cpu().numpy(), e


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_matches_single_boxes(prec):
    import torch

    from piny_b200.lib import DeviceBatch, DeviceBox
    boxes = _boxes()
    ref = [_single(S, pos, sp.nbeads, "fp64") for sp, pos, S in boxes]
    ctxs, d_pos, d_xm, d_f, hm = [], [], [], [], []
    keep = []
    for sp, pos, S in boxes:
        b = DeviceBox(S, sp.nbeads, prec)
        xmod = pos.mean(axis=0) if sp.nbeads > 1 else None
        b.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
        d = torch.from_numpy(pos).to("cuda:0")
        dx = torch.from_numpy(xmod).to("cuda:0") if xmod is not None else None
        f = torch.zeros_like(d)
        keep += [d, dx, f]
        ctxs.append(b)
        d_pos.append(d.data_ptr())
        d_xm.append(None if dx is None else dx.data_ptr())
        d_f.append(f.data_ptr())
        hm.append(S["hmat"])
    torch.cuda.synchronize()
    batch = DeviceBatch(ctxs)
    tol = 1e-12 if prec == "fp64" else 1e-5
    etol = 1e-11 if prec == "fp64" else 1e-6
    for call in range(2):  # capture, then replay of the graph
        es = batch.energy_force_device(d_pos, d_xm, hm, d_f)
        torch.cuda.synchronize()
        for i, (sp, pos, S) in enumerate(boxes):
            f = keep[3 * i + 2].cpu().numpy()
            assert rel_rms(f, ref[i][1]) < tol, (call, i)
            e0 = ref[i][2]
            scale = abs(e0["vvdw"]) + abs(e0["vcoul"]) + abs(e0["vrecip"]) + abs(e0["vself"])
            assert abs(es[i]["vintert"] - e0["vintert"]) <= etol * scale
            assert abs(es[i]["vintrat"] - e0["vintrat"]) <= etol * max(1.0, abs(e0["vintrat"]))
    assert batch.last_ms() > 0
    # a changed cell is a new graph; an unchanged call replays
    hm2 = [h * 1.001 for h in hm]
    es2 = batch.energy_force_device(d_pos, d_xm, hm2, d_f)
    assert all(np.isfinite(e["vintert"]) for e in es2)
    batch.close()
    for b in ctxs:
        b.close()
    for r in ref:
        r[0].close()


def test_batch_keeps_the_faster_form():
    """Without a form asked for, a batch the multi-box kernels cover is
    captured in both forms and the faster kept: either form is valid, the
    mode query names it, and the forces equal the one-box path."""
    import torch

    from piny_b200.lib import DeviceBatch, DeviceBox
    boxes = _boxes(nbox=6, seed=33)
    ctxs, d_pos, d_xm, d_f, hm, keep = [], [], [], [], [], []
    for sp, pos, S in boxes:
        b = DeviceBox(S, sp.nbeads, "mixed")
        xmod = pos.mean(axis=0) if sp.nbeads > 1 else None
        b.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
        d = torch.from_numpy(pos).to("cuda:0")
        dx = torch.from_numpy(xmod).to("cuda:0") if xmod is not None else None
        f = torch.zeros_like(d)
        keep += [d, dx, f]
        ctxs.append(b)
        d_pos.append(d.data_ptr())
        d_xm.append(None if dx is None else dx.data_ptr())
        d_f.append(f.data_ptr())
        hm.append(S["hmat"])
    batch = DeviceBatch(ctxs)
    batch.energy_force_device(d_pos, d_xm, hm, d_f)
    fused, nk = batch.last_mode()
    assert nk > 0 and (nk <= 48 if fused else nk > 4 * len(boxes))
    torch.cuda.synchronize()
    for i, (sp, pos, S) in enumerate(boxes):
        b0, f0, _ = _single(S, pos, sp.nbeads, "fp64")
        b0.close()
        assert rel_rms(keep[3 * i + 2].cpu().numpy(), f0) < 1e-5, i
    batch.close()
    for b in ctxs:
        b.close()


def test_every_launch_shape_gives_the_same_forces():
    boxes = _boxes(nbox=2, seed=5)
    for sp, pos, S in boxes:
        b0, f0, e0 = _single(S, pos, sp.nbeads, "fp64")
        b0.close()
        for choice in ([8, 0, 4, 0], [16, 1, 32, 1], [8, 1, 8, 1], [16, 0, 16, 0]):
            if choice[0] == 16 and min(S["ngrid_a"], S["ngrid_b"], S["ngrid_c"]) < 16:
                continue
            b, f, e = _single(S, pos, sp.nbeads, "fp64", choice)
            assert b.tuning() == choice
            assert rel_rms(f, f0) < 1e-12, choice
            assert abs(e["vintert"] - e0["vintert"]) <= 1e-11 * max(1.0, abs(e0["vintert"]))
            b.close()


def test_autotune_picks_a_valid_shape_and_remembers_it():
    import torch

    from piny_b200.lib import DeviceBox, PinyError
    sp, pos, S = _boxes(nbox=1, seed=9)[0]
    P = sp.nbeads
    box = DeviceBox(S, P, "mixed")
    xmod = pos.mean(axis=0) if P > 1 else None
    box.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
    d = torch.from_numpy(pos).to("cuda:0")
    dx = torch.from_numpy(xmod).to("cuda:0") if xmod is not None else None
    choice, ms = box.autotune(d.data_ptr(), None if dx is None else dx.data_ptr(), S["hmat"], reps=2, again=True)
    assert choice[0] in (8, 16) and choice[1] in (0, 1, 2) and choice[2] in (4, 8, 16, 32) and choice[3] in (0, 1)
    assert ms > 0
    assert box.tuning() == choice
    # a second context of the same shape applies the remembered result
    box2 = DeviceBox(S, P, "mixed")
    box2.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
    choice2, ms2 = box2.autotune(d.data_ptr(), None if dx is None else dx.data_ptr(), S["hmat"])
    assert choice2 == choice and ms2 == -1.0
    with pytest.raises(PinyError, match="ERR_ARG"):
        box2.set_tuning([12, 0, 8, 1])
    box.close()
    box2.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_c4_set_matches_oracle_box_by_box(prec, oracle):
    """The full 64-box uneven set of the batched benchmark (64-2048
    molecules, 1-64 beads, 16^3-64^3 meshes), autotuned, in one graph launch:
    every box's pair set equals the oracle's bit for bit and the forces of
    its first and last bead match the oracle's within 1e-12 (FP64) / 1e-5
    (MIXED) relative RMS; energies of boxes with at most 8 beads (the oracle
    evaluates all their beads) within 1e-11 relative / 1e-6 of the terms.
    MIXED runs the multi-box kernels, FP64 one graph branch per box."""
    import torch

    from helpers import pair_hash
    from piny_b200 import system, water
    from piny_b200.lib import DeviceBatch, DeviceBox

    specs = water.c4_specs()
    assert len(specs) == 64
    boxes, keep, d_pos, d_xm, d_f, hm = [], [], [], [], [], []
    for sp in specs:
        pos = water.build_positions(sp) / water.BOHR
        S = system.build_system(sp, pos)
        xmod = pos.mean(axis=0) if sp.nbeads > 1 else None
        b = DeviceBox(S, sp.nbeads, prec)
        n = b.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
        pi, pj = oracle.verlist(S, pos[0], xmod, S["hmat"], S["cutskin2"])
        gi, gj = b.get_list()
        assert n == len(pi) and pair_hash(gi, gj) == pair_hash(pi, pj)
        d = torch.from_numpy(pos).to("cuda:0")
        dx = torch.from_numpy(xmod).to("cuda:0") if xmod is not None else None
        f = torch.zeros_like(d)
        b.autotune(d.data_ptr(), None if dx is None else dx.data_ptr(), S["hmat"], reps=1)
        keep += [d, dx, f]
        boxes.append((sp, pos, S, xmod, pi, pj, b))
        d_pos.append(d.data_ptr())
        d_xm.append(None if dx is None else dx.data_ptr())
        d_f.append(f.data_ptr())
        hm.append(S["hmat"])
    torch.cuda.synchronize()
    batch = DeviceBatch([bx[-1] for bx in boxes])
    tol = {"fp64": 1e-12, "mixed": 1e-5}[prec]
    etol = {"fp64": 1e-11, "mixed": 1e-6}[prec]
    for call in range(2):  # capture, then replay of the graph
        # MIXED: the multi-box kernels (the form the capture keeps for this set)
        es = batch.energy_force_device(d_pos, d_xm, hm, d_f, kernels=(prec == "mixed"))
        assert batch.last_mode()[0] == (prec == "mixed")
        torch.cuda.synchronize()
        for i, (sp, pos, S, xmod, pi, pj, b) in enumerate(boxes):
            P = sp.nbeads
            f = keep[3 * i + 2].cpu().numpy()
            if call == 0 and P <= 8:
                fref, eref = oracle.energy_force(S, pos, xmod, S["hmat"], pi, pj)
                scale = 1.0
                if prec == "mixed":
                    scale = abs(eref["vvdw"]) + abs(eref["vcoul"]) + abs(eref["vrecip"]) + abs(eref["vself"])
                assert abs(es[i]["vintert"] - eref["vintert"]) <= etol * max(scale, abs(eref["vintert"])), i
                assert abs(es[i]["vintrat"] - eref["vintrat"]) <= etol * max(1.0, abs(eref["vintrat"])), i
                assert rel_rms(f, fref) < tol, (call, i)
            else:
                beads = [0, P - 1] if P > 1 else [0]
                fref, _ = oracle.energy_force(S, pos[beads], xmod, S["hmat"], pi, pj)
                assert rel_rms(f[beads], fref) < tol, (call, i)
    batch.close()
    for bx in boxes:
        bx[-1].close()


def test_mixed_pair_kernels_agree_with_fp64():
    """MIXED: the unrolled molecule-pair kernel (pair choice 0), the
    per-table molecule-pair kernel (2) and the site-list kernel (1) all give
    the FP64 forces within 1e-5 relative RMS."""
    boxes = _boxes(nbox=2, seed=5)
    for sp, pos, S in boxes:
        b0, f0, e0 = _single(S, pos, sp.nbeads, "fp64")
        b0.close()
        for choice in ([16, 0, 6, 1], [8, 2, 16, 0], [8, 1, 8, 1]):
            if choice[0] == 16 and min(S["ngrid_a"], S["ngrid_b"], S["ngrid_c"]) < 16:
                choice = [8] + choice[1:]
            b, f, e = _single(S, pos, sp.nbeads, "mixed", choice)
            assert b.tuning() == choice
            assert rel_rms(f, f0) < 1e-5, choice
            scale = abs(e0["vvdw"]) + abs(e0["vcoul"]) + abs(e0["vrecip"]) + abs(e0["vself"])
            assert abs(e["vintert"] - e0["vintert"]) <= 1e-6 * scale
            b.close()


@pytest.mark.parametrize("flags", [{}, {"energy": False}, {"distribute_ghosts": True}])
def test_batch_kernels_match_branches(flags):
    """The multi-box kernels (one persistent launch per phase and shape
    group) and one graph branch per box give the same MIXED forces (1e-5
    relative RMS of each box, and against the FP64 one-box path) and
    energies; the multi-box graph holds a few dozen launches, not one set per
    box.  Boxes of 1-64 beads on 16^3 and 32^3 meshes, so that several bead
    groups, tile edges and FFT lengths share a call."""
    import torch

    from piny_b200.lib import DeviceBatch, DeviceBox
    boxes = _boxes(nbox=12, seed=33)
    ctxs, d_pos, d_xm, hm, keep = [], [], [], [], []
    for sp, pos, S in boxes:
        b = DeviceBox(S, sp.nbeads, "mixed")
        xmod = pos.mean(axis=0) if sp.nbeads > 1 else None
        b.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
        d = torch.from_numpy(pos).to("cuda:0")
        dx = torch.from_numpy(xmod).to("cuda:0") if xmod is not None else None
        keep += [d, dx]
        ctxs.append(b)
        d_pos.append(d.data_ptr())
        d_xm.append(None if dx is None else dx.data_ptr())
        hm.append(S["hmat"])
    f_fused = [torch.zeros_like(keep[2 * i]) for i in range(len(boxes))]
    f_branch = [torch.zeros_like(keep[2 * i]) for i in range(len(boxes))]
    batch = DeviceBatch(ctxs)
    energy = flags.get("energy", True)
    ghosts = flags.get("distribute_ghosts", False)
    for call in range(2):
        ef = batch.energy_force_device(d_pos, d_xm, hm, [f.data_ptr() for f in f_fused], energy=energy,
                                       distribute_ghosts=ghosts, kernels=True)
        fused, nk = batch.last_mode()
        assert fused and 0 < nk <= 48, (fused, nk)
        eb = batch.energy_force_device(d_pos, d_xm, hm, [f.data_ptr() for f in f_branch], energy=energy,
                                       distribute_ghosts=ghosts, branches=True)
        fused_b, nkb = batch.last_mode()
        assert not fused_b and nkb > 4 * len(boxes)
        torch.cuda.synchronize()
        for i, (sp, pos, S) in enumerate(boxes):
            a, b = f_fused[i].cpu().numpy(), f_branch[i].cpu().numpy()
            assert rel_rms(a, b) < 1e-5, (call, i)
            if energy:
                scale = abs(eb[i]["vvdw"]) + abs(eb[i]["vcoul"]) + abs(eb[i]["vrecip"]) + abs(eb[i]["vself"])
                assert abs(ef[i]["vintert"] - eb[i]["vintert"]) <= 1e-6 * scale, i
                assert abs(ef[i]["vintrat"] - eb[i]["vintrat"]) <= 1e-9 * max(1.0, abs(eb[i]["vintrat"])), i
                assert np.allclose(ef[i]["pvten"], eb[i]["pvten"], rtol=1e-5, atol=1e-6 * scale)
    if not ghosts:
        for i, (sp, pos, S) in enumerate(boxes[:3]):
            b0, f0, _ = _single(S, pos, sp.nbeads, "fp64")
            b0.close()
            assert rel_rms(f_fused[i].cpu().numpy(), f0) < 1e-5, i
    batch.close()
    for b in ctxs:
        b.close()


def test_batch_tune_keeps_a_shape_set_that_gives_the_same_forces():
    """DeviceBatch.tune times the batch with every box's own autotuned
    launch shape and with the defaults, keeps the faster set, and the
    forces stay those of the one-box FP64 path (MIXED tolerance)."""
    import torch

    from piny_b200.lib import DeviceBatch, DeviceBox
    boxes = _boxes(nbox=5, seed=21)
    ctxs, d_pos, d_xm, d_f, hm, keep = [], [], [], [], [], []
    for sp, pos, S in boxes:
        b = DeviceBox(S, sp.nbeads, "mixed")
        xmod = pos.mean(axis=0) if sp.nbeads > 1 else None
        b.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
        d = torch.from_numpy(pos).to("cuda:0")
        dx = torch.from_numpy(xmod).to("cuda:0") if xmod is not None else None
        f = torch.zeros_like(d)
        keep += [d, dx, f]
        ctxs.append(b)
        d_pos.append(d.data_ptr())
        d_xm.append(None if dx is None else dx.data_ptr())
        d_f.append(f.data_ptr())
        hm.append(S["hmat"])
    batch = DeviceBatch(ctxs)
    times, kept = batch.tune(d_pos, d_xm, hm, d_f, reps=2)
    assert set(times) == {"per_box", "defaults", "defaults_own_tiles"} and kept in times
    assert all(t > 0 for t in times.values())
    assert times[kept] == min(times.values())
    batch.energy_force_device(d_pos, d_xm, hm, d_f)
    torch.cuda.synchronize()
    for i, (sp, pos, S) in enumerate(boxes):
        b0, f0, _ = _single(S, pos, sp.nbeads, "fp64")
        b0.close()
        assert rel_rms(keep[3 * i + 2].cpu().numpy(), f0) < 1e-5, i
    batch.close()
    for b in ctxs:
        b.close()
