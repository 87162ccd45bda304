#!/usr/bin/env python
"""Benchmark: bead-force evaluations per second of the flexible-water force
path (q-TIP4P/F, 4096 molecules, 32 beads, PME 64^3 order 8) in mixed
precision on B200, against the FP64 device path and PINY's own CPU path.

A step is one evaluation of forces, energies and virial of all 32 beads of
the box at a fixed Verlet list (the list build is timed and reported apart).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU runs (torchrun, one rank per GPU) hold one box replica per GPU
(weak scaling); the only cross-rank traffic is the barrier and the max-reduce
of the timing.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "bead-force evals/s (TIP4P/F 4096 mol x 32 beads) mixed vs FP64 GPU, rel err <= 1e-5"
UNIT = "bead-force evals/s"
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="tip4pf_4096_p32",
                    help="a named box; c4_batch64: 64 uneven boxes in one graph launch per step; "
                         "c5_grad: parameter gradients of 1024 TIP4P/F x 16 beads; "
                         "pimd_nvt: PINY's NVT ring-polymer MD step of 4096 TIP4P/F x 32 beads; "
                         "respa: the force calls of one PINY RESPA step (respa_steps_lrf 2, respa_steps_intra 2) "
                         "of 4096 TIP4P/F x 32 beads; pimd_nvt_respa: the NVT PIMD step with those RESPA loops; "
                         "list_<N>: Verlet-list builds of N TIP4P/F molecules x 4 beads, link cells and sweep")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-energy", action="store_true", help="forces only (PINYB200_NO_ENERGY), for profiling")
    ap.add_argument("--fd", action="store_true", help="c5_grad: also check against central differences")
    ap.add_argument("--batch-branches", action="store_true",
                    help="c4_batch: one graph branch per box (no timing of the two forms)")
    ap.add_argument("--profile-step", action="store_true",
                    help="c4_batch: one extra step between cudaProfilerStart/Stop (ncu --profile-from-start off)")
    ap.add_argument("--batch-kernels", action="store_true",
                    help="c4_batch: the multi-box kernels (no timing of the two forms)")
    ap.add_argument("--tuning", default="", help="pin a launch shape: tile,pair_kernel,blocks_per_sm,overlap")
    return ap.parse_args()


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def metric_for(config, spec):
    """The metric a single-box line reports: the headline metric for the
    4096 x 32 box, the same quantity named for its box otherwise."""
    if config == "tip4pf_4096_p32":
        return METRIC
    return "bead-force evals/s (%s %d mol x %d beads)" % (spec.model.name, spec.nmol, spec.nbeads)


def cpu_info():
    """Host CPU model and logical core count (for the CPU baselines)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "host_cores": os.cpu_count()}


def piny_golden(name):
    """PINY's own evaluation of a benchmark box, when tests/golden holds it:
    (fixture, bead positions and mode-1 positions PINY used, in Bohr) --
    the seeded generator's positions moved by the stored ulp offsets."""
    from piny_b200 import water
    path = os.path.join(ROOT, "tests", "golden", name + ".npz")
    if not os.path.exists(path):
        return None
    F = dict(np.load(path))
    if "pos" in F:  # a fixture that holds the positions themselves (every bead)
        F["ref_beads"] = np.arange(F["pos"].shape[0])
        return F, F["pos"], F.get("xmod")
    gen = water.build_positions(water.named_spec(name)) / water.BOHR
    pos = (gen.view(np.int64) + F["pos_ulp"].astype(np.int64)).view(np.float64)
    xmod = None
    if "xmod_ulp" in F:
        xmod = (gen.mean(axis=0).view(np.int64) + F["xmod_ulp"].astype(np.int64)).view(np.float64)
    return F, pos, xmod


def kernel_bytes(S, P, precision, npairs, nmolp):
    """Algorithmic bytes of one launch of each kernel of an evaluation (all
    P beads): what the kernel must read and write at least, given the data
    layout (FP64 positions and forces [site][xyz][bead]; a real PME grid of
    4 (MIXED) or 8 (FP64) bytes per point; half spectrum; per (charge, bead)
    PME records of 32 / 48 bytes plus a 4-byte bin entry)."""
    N, G = int(S["natm"]), int(S["ngrid_a"]) * int(S["ngrid_b"]) * int(S["ngrid_c"])
    nq = int(np.count_nonzero(S["charge"]))
    rb = 4 if precision == "mixed" else 8
    rec = 32 if precision == "mixed" else 48
    nrec = nq * P
    spec = (int(S["ngrid_a"]) // 2 + 1) * int(S["ngrid_b"]) * int(S["ngrid_c"]) * 2 * rb * P
    nb, nbe, nec = int(S.get("nbond", 0)), int(S.get("nbend", 0)), int(S.get("necor", 0))
    return {
        "transpose_in": 48.0 * N * P,
        "ghost_pos": 96.0 * int(S.get("nghost", 0)) * P,
        # positions in, forces out, the shared list once (the scope table's pair figure)
        "pair": 48.0 * N * P + 4.0 * npairs,
        "pme_grid_clear (memset)": float(G * P * rb),
        "pme_bin": nrec * (24.0 + rec + 4.0),
        "pme_spread": nrec * (rec + 4.0) + G * P * rb,
        "pme_plane_fwd": float(G * P * rb + spec),
        "pme_conv_c": 2.0 * spec,
        "pme_plane_inv": float(spec + G * P * rb),
        "pme_gather": G * P * rb + nrec * (rec + 4.0 + 24.0),
        "pme_force_add": 72.0 * nrec,
        "intra (bond, bend, ecor)": 72.0 * P * (2 * nb + 3 * nbe + 2 * nec),
        "transpose_out": 48.0 * N * P,
    }


def kernel_profile(box, step, S, P, precision, npairs, nmolp, flush, stream, reps=5):
    """Serialised per-kernel times of `reps` evaluations (CUDA events after
    every kernel, pinyb200_set_kernel_timing; L2 flushed before each), the
    median per kernel with its algorithmic bytes and HBM fraction."""
    import torch
    hbm, _ = peaks()
    box.set_kernel_timing(True)
    step()
    torch.cuda.synchronize()
    runs = []
    for _ in range(reps):
        flush.zero_()
        step()
        torch.cuda.synchronize()
        runs.append(box.kernel_times())
    box.set_kernel_timing(False)
    kb = kernel_bytes(S, P, precision, npairs, nmolp)
    out = []
    for i, (name, _) in enumerate(runs[0]):
        ms = float(np.median([r[i][1] for r in runs]))
        b = kb.get(name)
        gbs = b / (ms * 1e-3) / 1e9 if b and ms > 0 else None
        out.append({"kernel": name, "ms": ms, "algorithmic_bytes": b, "achieved_GBs": gbs,
                    "hbm_frac": gbs / hbm if gbs else None})
    tot = sum(k["ms"] for k in out)
    for k in out:
        k["share"] = k["ms"] / tot if tot > 0 else None
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)

        def reader():
            for line in self.proc.stdout:
                self.lines.append(line.strip())
        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# PINY's own CPU path (oracle/_ref/piny_ref, built from the PINY sources)

def piny_ref_binary():
    p = os.path.join(ROOT, "oracle", "_ref", "piny_ref")
    return p if os.path.exists(p) else None


def time_piny_cpu(spec, pos_A, nproc, beads_per_proc, reps):
    """Run ``nproc`` independent PINY processes on copies of the box, each
    evaluating ``beads_per_proc`` beads per step (PINY's serial bead loop),
    ``reps`` timed steps after one warm-up.  Returns per-step bead-evals/s."""
    from piny_b200 import water
    exe = piny_ref_binary()
    tmp = tempfile.mkdtemp(prefix="piny_cpu_")
    dirs = []
    for k in range(nproc):
        d = os.path.join(tmp, "r%d" % k)
        water.write_piny_input(d, spec, pos_A)
        dirs.append(d)
    procs = [subprocess.Popen([exe, "time", d, "water.input", str(reps), str(beads_per_proc)],
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True) for d in dirs]
    per = []
    for p in procs:
        out, err = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("piny_ref failed: " + err[-400:])
        per.append([float(l.split()[3]) for l in out.splitlines() if l.startswith("time")])
    shutil.rmtree(tmp, ignore_errors=True)
    per = np.array(per)  # [proc][rep]
    step_s = per.max(axis=0)
    return nproc * beads_per_proc / step_s, step_s


def piny_bead_seconds(specs, reps=3, workers=None):
    """Seconds per bead-force evaluation of PINY's CPU path for each box of
    `specs` (oracle/_ref/piny_ref, 1 bead, median of `reps` after its
    warm-up), the boxes run as concurrent single-threaded processes, at most
    `workers` (default: every host core) at a time."""
    from piny_b200 import water
    exe = piny_ref_binary()
    workers = workers or (os.cpu_count() or 1)
    tmp = tempfile.mkdtemp(prefix="piny_cpu_")
    out = [None] * len(specs)
    running = []
    todo = list(range(len(specs)))
    # largest boxes first, so the pool drains evenly
    todo.sort(key=lambda i: -specs[i].nmol)
    while todo or running:
        while todo and len(running) < workers:
            i = todo.pop(0)
            d = os.path.join(tmp, "b%d" % i)
            water.write_piny_input(d, specs[i], water.build_positions(specs[i]))
            running.append((i, subprocess.Popen([exe, "time", d, "water.input", str(reps), "1"],
                                                stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        i, p = running.pop(0)
        o, e = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("piny_ref failed: " + e[-300:])
        out[i] = float(np.median([float(l.split()[3]) for l in o.splitlines() if l.startswith("time")]))
    shutil.rmtree(tmp, ignore_errors=True)
    return np.array(out)


def time_oracle_port(S, pos_bohr, xmod, beads):
    from oracle.oracle import Oracle
    O = Oracle()
    pi, pj = O.verlist(S, pos_bohr[0], xmod, S["hmat"], S["cutskin2"])
    t = time.perf_counter()
    O.energy_force(S, pos_bohr[:beads], xmod, S["hmat"], pi, pj)
    dt = time.perf_counter() - t
    return beads / dt, dt


def cpu_baseline(spec, pos_A, pos_bohr, S, xmod, reps=5):
    """PINY's CPU path on one host core: a bounded sample of the box (at most
    2 of its beads per step), the median of `reps` steps after one warm-up,
    scaled per bead-force evaluation."""
    nb = min(2, spec.nbeads)
    if piny_ref_binary():
        rate, steps = time_piny_cpu(spec, pos_A, nproc=1, beads_per_proc=nb, reps=reps)
        return {"value": float(np.median(rate)), "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "PINY energy_control sub-steps (oracle/_ref/piny_ref) on %d of %d beads per step, "
                          "1 host core, median of %d steps after 1 warm-up" % (nb, spec.nbeads, reps),
                "step_s": [float(x) for x in steps], **cpu_info()}
    rate, dt = time_oracle_port(S, pos_bohr, xmod, 1)
    return {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "oracle restatement, 1 of %d beads, 1 host core" % spec.nbeads, **cpu_info()}


def box_config(spec, args, natm, grid, npairs=None, list_s=None):
    """The config object of a single-box line (both arms print the same)."""
    return {"workload": args.config, "molecules": spec.nmol, "sites": natm, "beads": spec.nbeads,
            "box_A": spec.L, "pme_grid": grid, "pme_order": spec.order, "cutoff_A": spec.cutoff,
            "precision": args.precision, "verlet_pairs": npairs, "list_build_s": list_s,
            "l2": "256 MiB buffer written between timed steps; per-step CUDA events on the launch stream",
            "parallelism": "replica per GPU" if args.gpus > 1 else "single GPU"}


def run_reference(args, ws, rank):
    """--impl reference: PINY's own CPU path on all host cores."""
    if rank != 0:
        return 0
    from piny_b200 import water
    if piny_ref_binary() is not None and (args.config.startswith("c4_batch") or args.config == "c5_grad"):
        return run_reference_sampled(args)
    if args.config not in ("tip4pf_4096_p32", "tip4pf_1024_p16", "tip4pf_1024_p32", "spcfw_256_p1",
                           "spcfw_256_p32", "tip4pf_256_p4", "spcfw_216_p4"):
        print(json.dumps({"impl": "reference", "unavailable": "no PINY CPU arm for the %s workload "
                                                              "(PINY has no device-side MD step)" % args.config}))
        return 0
    spec = water.named_spec(args.config)
    if piny_ref_binary() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/piny_ref not built (needs the PINY "
                                                                "sources at build time)"}))
        return 0
    from piny_b200 import system
    pos_A = water.build_positions(spec)
    S = system.build_system(spec, pos_A / water.BOHR)
    ncpu = os.cpu_count() or 1
    nproc = max(1, min(ncpu, spec.nbeads))
    warm = max(3, args.warmup)
    # piny_ref makes one warm-up evaluation itself; the rest are dropped here
    rate, steps = time_piny_cpu(spec, pos_A, nproc=nproc, beads_per_proc=1, reps=max(1, args.steps) + warm - 1)
    rate, steps = rate[warm - 1:], steps[warm - 1:]
    value = float(np.mean(rate))
    line = {
        "impl": "reference", "metric": metric_for(args.config, spec), "value": value, "unit": UNIT, "n_gpus": 0,
        "steps": args.steps, "warmup": warm, "ms_per_step": float(np.mean(steps)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": box_config(spec, args, int(S["natm"]), int(S["ngrid_a"])),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "reference",
                         "sample": "%d PINY processes (oracle/_ref/piny_ref) x 1 bead per step, one per host "
                                   "core, the box's list fixed; a step is %d of the box's %d bead "
                                   "evaluations" % (nproc, nproc, spec.nbeads), **cpu_info()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_reference_sampled(args):
    """--impl reference for the batched and the gradient workloads: PINY's
    CPU path, one bead of each box per host process, every host core.
    c4_batch64: per step every bead of the 64 boxes; the step time is the
    per-bead seconds of each box times its beads, spread over the cores.
    c5_grad: the gradient by central differences, 2 x 9 + 1 evaluations of
    the 16-bead box per gradient, spread over the cores."""
    from piny_b200 import system, water
    ncpu = os.cpu_count() or 1
    warm = max(3, args.warmup)
    if args.config.startswith("c4_batch"):
        nbox = int(args.config[len("c4_batch"):] or 64)
        specs = water.c4_specs(nbox=nbox, seed=2024)
        t = piny_bead_seconds(specs, reps=max(3, min(args.steps, 5)))
        work = float(np.sum([sp.nbeads * t[i] for i, sp in enumerate(specs)]))
        nbead = sum(sp.nbeads for sp in specs)
        step_s = work / ncpu
        value, unit = nbead / step_s, UNIT
        metric = "bead-force evals/s (64 uneven TIP4P/F boxes, batched)"
        sample = ("PINY (oracle/_ref/piny_ref): 1 bead of each of the %d boxes, median of its steps after a "
                  "warm-up, boxes as concurrent single-threaded processes; a step = every bead of every box, "
                  "the summed seconds spread over %d cores" % (nbox, ncpu))
        cfg = {"workload": args.config, "boxes": nbox, "bead_evals_per_step": nbead,
               "molecules": [sp.nmol for sp in specs], "beads": [sp.nbeads for sp in specs],
               "pme_grid": [sp.grid for sp in specs], "precision": args.precision}
    else:
        spec = water.named_spec("tip4pf_1024_p16")
        t = piny_bead_seconds([spec], reps=max(3, min(args.steps, 5)))[0]
        nev = 2 * 9 + 1
        step_s = nev * spec.nbeads * t / min(ncpu, nev * spec.nbeads)
        value, unit = 1.0 / step_s, "gradient evals/s"
        metric = ("parameter-gradient evals/s (9 q-TIP4P/F parameters; energy + force-matching loss; "
                  "1024 mol x 16 beads)")
        sample = ("PINY (oracle/_ref/piny_ref) has no gradient: central differences, %d evaluations of the "
                  "16-bead box per gradient, from PINY's seconds per bead (median after a warm-up), spread "
                  "over %d cores" % (nev, min(ncpu, nev * spec.nbeads)))
        cfg = {"workload": "c5_grad", "molecules": spec.nmol, "beads": spec.nbeads, "pme_grid": spec.grid,
               "parameters": 9}
    line = {"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": 0, "steps": args.steps,
            "warmup": warm, "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": unit, "cores": ncpu, "kind": "reference", "sample": sample,
                             **cpu_info()},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def list_timing(S, P, ns, pos, xmod, precision, dev, reps=5, methods=None):
    """Verlet-list builds of one box: the host call pinyb200_build_list
    (wall time, median of reps after one) and device rebuilds
    (pinyb200_update_list_device, CUDA events on the stream, median) with
    the molecules moved rigidly between calls so that each one rebuilds,
    per list method (link cells / sweep)."""
    import torch

    from piny_b200 import lib
    from piny_b200.lib import DeviceBox
    rng = np.random.default_rng(3)
    natm = int(S["natm"])
    # rigid molecule moves: one random vector per molecule of ns consecutive sites
    mol_of = np.arange(natm) // ns
    shift = rng.normal(scale=0.4, size=(natm // ns, 3))[mol_of]
    p2 = pos + shift[None]
    d0 = torch.from_numpy(pos).to(dev)
    d2 = torch.from_numpy(p2).to(dev)
    x0 = torch.from_numpy(np.ascontiguousarray(pos.mean(axis=0))).to(dev)
    x2 = torch.from_numpy(np.ascontiguousarray(p2.mean(axis=0))).to(dev)
    # the rebuild is enqueued without a host wait: time it on a stream of its own
    stream = torch.cuda.Stream(dev)
    torch.cuda.synchronize()
    out = {}
    for method, name in ((lib.LIST_LNK, "lnk"), (lib.LIST_NOLST, "nolst")):
        if methods and name not in methods:
            continue
        box = DeviceBox(S, P, precision)
        box.set_list_method(method)
        host = []
        for k in range(reps + 1):
            t0 = time.perf_counter()
            npairs = box.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
            host.append(time.perf_counter() - t0)
        cells, _ = box.list_cells()
        sp0 = box.check_list_device(d0.data_ptr(), 0.0)[2]
        box.list_set_spread(sp0)
        dev_ms, used = [], []
        for k in range(2 * reps + 1):
            d, x = (d2, x2) if k % 2 == 0 else (d0, x0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            box.update_list_device(d.data_ptr(), x.data_ptr(), S["hmat"], stream=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            if k:
                dev_ms.append(e0.elapsed_time(e1))
                used.append(box.list_cells()[1])
        st = box.list_status(stream=stream.cuda_stream)
        out[name] = {"host_build_ms": 1e3 * float(np.median(host[1:])), "device_rebuild_ms": float(np.median(dev_ms)),
                     "device_rebuilds": int(st["rebuilds"]), "cells": list(cells),
                     "cells_used_on_device": bool(all(used)), "npairs": int(npairs)}
        box.close()
    return out


def run_list(args, ws, rank, local):
    """--config list_<N>: list builds of N TIP4P/F molecules x 4 beads;
    list_<named box>: of that box (e.g. list_tip4pf_4096_p32)."""
    import torch

    from piny_b200 import system, water
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    what = args.config[len("list_"):]
    if what.isdigit():
        nmol = int(what)
        spec = water.BoxSpec(water.TIP4P_F, nmol, water.density_box_edge(nmol), 4, 298.0, 7, grid=32, order=6)
    else:
        spec = water.named_spec(what)
        nmol = spec.nmol
    pos = water.build_positions(spec) / water.BOHR
    S = system.build_system(spec, pos)
    res = list_timing(S, spec.nbeads, spec.model.nsite, pos, pos.mean(axis=0), args.precision, dev,
                      reps=max(3, args.steps))
    if rank == 0:
        best = min(v["device_rebuild_ms"] for v in res.values())
        print(json.dumps({"metric": "Verlet-list device rebuilds/s (%s %d mol x %d beads)" %
                                    (spec.model.name, nmol, spec.nbeads),
                          "value": 1e3 / best, "unit": "rebuilds/s", "n_gpus": 1, "steps": max(3, args.steps),
                          "warmup": 1, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
                          "config": {"workload": "list build, %d %s molecules, %d beads, box %.1f A, "
                                                 "rigid molecule moves of 0.4 Bohr rms per component" %
                                                 (nmol, spec.model.name, spec.nbeads, spec.L)},
                          "methods": res}))
    return 0


def alg_bytes_per_bead_eval(S, P, nlist, precision):
    """Algorithmic bytes of one bead-force evaluation: FP64 positions in and
    forces out, the shared half list once per batch of beads, and six passes
    over the PME grid (spread, forward FFT read/write, inverse FFT
    read/write, gather)."""
    G = S["ngrid_a"] * S["ngrid_b"] * S["ngrid_c"]
    bg = 8 if precision == "mixed" else 16
    return 48.0 * S["natm"] + 4.0 * nlist / P + 6.0 * G * bg


def run_grad(args, ws, rank, local):
    """Gradients of the energy and of a force-matching loss with respect to
    the 9 q-TIP4P/F parameters (1024 molecules, 16 beads, 32^3 mesh): one
    step = forward evaluation + adjoint pass; MIXED timed, checked against
    the FP64 adjoint and against central differences of the FP64 device
    forward (h = 1e-5 relative)."""
    import dataclasses

    import torch

    from piny_b200 import params, water
    from piny_b200.params import PinyForceField

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    spec = water.named_spec("tip4pf_1024_p16")
    if ws > 1:
        spec = dataclasses.replace(spec, seed=spec.seed + rank)
    pos_A = water.build_positions(spec)
    theta = params.theta_of(spec.model)
    rng = np.random.default_rng(2024)
    theta_t = theta * (1.0 + rng.uniform(-0.02, 0.02, size=theta.shape))
    f64 = PinyForceField(spec, pos_A, "fp64", device=str(dev))
    _, f_target = f64.energy_forces(theta_t)
    E64, F64 = f64.energy_forces(theta)
    fbar = 2.0 * (F64 - f_target)
    g64 = f64.adjoint(theta, 1.0, fbar)
    mixed = PinyForceField(spec, pos_A, args.precision, device=str(dev))
    E, F = mixed.energy_forces(theta)
    d_fbar = torch.from_numpy(2.0 * (F - f_target)).to(dev)
    box = mixed.box
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        return box.grad(mixed.d_pos.data_ptr(), None if mixed.d_xmod is None else mixed.d_xmod.data_ptr(),
                        mixed.hmat, d_fbar.data_ptr(), stream=stream.cuda_stream)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if ws > 1:
        torch.distributed.barrier()
    ms_list = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dE, dF = step()
        e1.record(stream)
        e1.synchronize()
        ms_list.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    ms = float(np.mean(ms_list))
    if ws > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    g_mixed = dE + dF
    # end to end: positions in from pinned host memory, the gradient back
    pin = torch.empty(mixed.d_pos.shape, dtype=torch.float64).pin_memory()
    pin.copy_(mixed.d_pos.cpu())
    e2e_ms = []
    for k in range(args.steps + 2):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        mixed.d_pos.copy_(pin, non_blocking=True)
        step()
        e1.record(stream)
        e1.synchronize()
        if k >= 2:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e = float(np.mean(e2e_ms))
    npairs = box.list_info()["npairs"]
    alg = 2.0 * sum(kernel_bytes(mixed.S, spec.nbeads, args.precision, npairs, 0).values())
    hbm, peak_kind = peaks()
    c5_cpu = None
    if rank == 0 and not args.no_cpu_baseline and piny_ref_binary():
        try:
            tb = float(piny_bead_seconds([spec], reps=5, workers=1)[0])
            nev = 2 * len(theta) + 1
            c5_cpu = {"value": 1.0 / (nev * spec.nbeads * tb), "unit": "gradient evals/s", "cores": 1,
                      "kind": "reference",
                      "sample": "PINY (oracle/_ref/piny_ref) has no gradient: central differences take %d "
                                "evaluations of the 16-bead box; PINY's seconds per bead (1 bead, median of 5 "
                                "after a warm-up, 1 host core) x %d" % (nev, nev * spec.nbeads),
                      "seconds_per_bead": tb, **cpu_info()}
        except Exception as exc:  # reported, not fatal
            c5_cpu = {"value": None, "unit": "gradient evals/s", "cores": 1, "kind": "reference",
                      "sample": "failed: %s" % exc}
    rel_mixed = float(np.abs(g_mixed - g64).max() / np.abs(g64).max())
    fd = None
    if getattr(args, "fd", False):
        gfd = np.zeros(len(theta))
        for k in range(len(theta)):
            h = 1e-5 * abs(theta[k])
            tp, tm = theta.copy(), theta.copy()
            tp[k] += h
            tm[k] -= h
            Ep, Fp = f64.energy_forces(tp)
            Em, Fm = f64.energy_forces(tm)
            gfd[k] = (Ep - Em) / (2 * h) + (((Fp - f_target) ** 2).sum() - ((Fm - f_target) ** 2).sum()) / (2 * h)
        fd = {params.PARAMS[k]: {"adjoint_fp64": float(g64[k]), "central_difference": float(gfd[k]),
                                 "rel": float(abs(g64[k] - gfd[k]) / max(abs(gfd[k]), 1e-300))}
              for k in range(len(theta))}
    if rank == 0:
        line = {
            "metric": "parameter-gradient evals/s (9 q-TIP4P/F parameters; energy + force-matching loss; "
                      "1024 mol x 16 beads)", "value": ws * 1e3 / ms, "unit": "gradient evals/s",
            "n_gpus": ws, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64acc" if args.precision == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": "c5_grad", "molecules": spec.nmol, "beads": spec.nbeads, "pme_grid": spec.grid,
                       "parameters": list(params.PARAMS), "target": "theta perturbed by seeded +-2 %",
                       "step": "forward evaluation + adjoint (pinyb200_grad)",
                       "l2": "256 MiB buffer written between timed steps; CUDA events on the launch stream"},
            "gradient": {"theta": theta.tolist(), "mixed": g_mixed.tolist(), "fp64": g64.tolist(),
                         "max_rel_mixed_vs_fp64": rel_mixed, "finite_differences_fp64": fd},
            "roofline": {"bound": "hbm", "kernel": "gradient step (forward evaluation + adjoint)",
                         "achieved": alg / (ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                         "frac": alg / (ms * 1e-3) / 1e9 / hbm, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg,
                         "bytes_model": "twice the forward evaluation's per-kernel algorithmic bytes (the adjoint "
                                        "re-reads positions, list, grid and records the same way)"},
            "cpu_baseline": c5_cpu,
            "e2e": {"value": ws * 1e3 / e2e, "unit": "gradient evals/s",
                    "h2d_bytes_per_step": int(pin.numel() * 8), "d2h_bytes_per_step": int(2 * len(theta) * 8),
                    "ms_per_step": e2e},
            # forward evaluation, then u, ghost, pair, ecor, bond, bend adjoint
            # kernels and the PME adjoint (dipole spread, 3 FFT kernels, gather)
            "gpu_launches": (box_launches(mixed.S, spec.nbeads) + 12) * args.steps, "clocks": clocks,
        }
        print(json.dumps(line))
    f64.close()
    mixed.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_pimd(args, ws, rank, local):
    """PINY's NVT ring-polymer MD step on the device (pinyb200_pimd_step):
    4096 q-TIP4P/F x 32 beads, normal modes, chains of 4 on every
    coordinate, dt = 20 a.u.; a step is the chains and half kicks, the
    mode transforms, drift, springs, PINY's list test and (when due) list
    rebuild on the device, one force evaluation of all beads, and the force
    post-processing.  The transform kernel is timed alone for its HBM
    roofline."""
    import dataclasses

    import torch

    from piny_b200 import pimd, system, water
    from piny_b200 import respa as R
    from piny_b200.lib import NORMAL_MODES, TO_MODES, DeviceBox, DevicePimd, pimd_transform

    use_respa = args.config == "pimd_nvt_respa"
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    spec = water.named_spec("tip4pf_4096_p32")
    if ws > 1:
        spec = dataclasses.replace(spec, seed=spec.seed + rank)
    pos = water.build_positions(spec) / water.BOHR
    S = system.build_system(spec, pos)
    natm, P = int(S["natm"]), spec.nbeads
    ghost = np.zeros(natm, bool)
    ghost[np.asarray(S["ghost_atom"])] = True
    mass = np.tile(np.asarray(spec.model.masses, np.float64), spec.nmol) * 1822.888486
    dt = 20.0
    nres = (2, 1, 2, 1) if use_respa else (1, 1, 1, 1)
    if use_respa:
        dt = 20.0 * 4  # outer step of four 20 a.u. inner steps
    # with RESPA the chains run at every inner step (ix_respa 5): the bead
    # chains of 32 beads (tuned to the ring polymer's frequency) do not stay
    # stable over the 80 a.u. outer step
    ix_respa = 5 if use_respa else 1
    setup = pimd.nvt_setup(mass, ghost, P, NORMAL_MODES, spec.temperature, dt, 800.0, len_nhc=4, nyosh=3, nres=nres,
                           ix_respa=ix_respa)
    rng = np.random.default_rng(spec.seed)
    v = rng.normal(size=(P, natm, 3)) * np.sqrt(spec.temperature / water.BOLTZ / setup["bead_mass"])[:, :, None]
    v[:, ghost, :] = 0.0
    box = DeviceBox(S, P, args.precision)
    xmod0 = pos.mean(axis=0)
    box.build_list(pos[0], xmod0, S["hmat"], S["cutskin2"])
    if use_respa:
        box.set_respa(R.respa_setup(*nres, True, True, np.minimum(np.asarray(S["cutoff"]), 5.0 / water.BOHR),
                                    1.0 / water.BOHR, np.asarray(S["bond_eq"])))
    pm = DevicePimd(setup)
    stream = torch.cuda.current_stream(dev)
    d_x = torch.from_numpy(pos.copy()).to(dev)
    d_v = torch.from_numpy(v).to(dev)
    d_f = torch.zeros_like(d_x)
    pm.forces(box, d_x.data_ptr(), d_f.data_ptr(), S["hmat"], stream=stream.cuda_stream)
    # the list was built from these positions: their bead spread is the
    # reference of the device list test that every step runs
    box.list_set_spread(box.check_list_device(d_x.data_ptr(), 0.0, stream=stream.cuda_stream)[2])

    def step():
        return pm.step(box, d_x.data_ptr(), d_v.data_ptr(), d_f.data_ptr(), S["hmat"], stream=stream.cuda_stream)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if ws > 1:
        torch.distributed.barrier()
    ms_list = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e = step()
        e1.record(stream)
        e1.synchronize()
        ms_list.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    ms = float(np.mean(ms_list))
    rebuilds = box.list_status(stream=stream.cuda_stream)["rebuilds"]
    # the force evaluation alone on the same positions (the steps replay a
    # CUDA graph, which records no per-phase events)
    d_xm = torch.from_numpy(np.ascontiguousarray(d_x.cpu().numpy().mean(axis=0))).to(dev)
    d_ft = torch.empty_like(d_f)
    force_ms = []
    for r in range(8):
        box.energy_force_device(d_x.data_ptr(), d_xm.data_ptr(), S["hmat"], d_ft.data_ptr(), stream=stream.cuda_stream,
                                distribute_ghosts=True)
        if r >= 3:
            force_ms.append(box.last_timing()[0])
    # the transform alone: positions -> modes of all beads (HBM roofline)
    tr = torch.empty_like(d_x)
    tr.copy_(d_x)
    tms = []
    for r in range(13):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pimd_transform(tr.data_ptr(), natm, P, NORMAL_MODES, TO_MODES, stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        if r >= 3:
            tms.append(e0.elapsed_time(e1))
    t_ms = float(np.mean(tms))
    t_bytes = 2.0 * P * natm * 3 * 8
    if ws > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    hbm, peak_kind = peaks()
    if rank == 0:
        inner = int(np.prod(nres))
        line = {
            "metric": ("PIMD NVT RESPA steps/s (TIP4P/F 4096 mol x 32 beads, normal modes, 4 inner steps)"
                       if use_respa else "PIMD NVT steps/s (TIP4P/F 4096 mol x 32 beads, normal modes)"),
            "value": ws * 1e3 / ms,
            "unit": "MD steps/s", "n_gpus": ws, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (step) + " + ("f32+f64acc" if args.precision == "mixed" else "f64") + " (forces)",
            "data": "synthetic",
            "config": {"workload": args.config, "molecules": spec.nmol, "beads": P, "dt_au": dt,
                       "respa": {"nres_ter_tor_tra_pimd": list(nres), "ix_respa": ix_respa, "cutoff_res_A": 5.0,
                                 "rheal_A": 1.0, "inner_dt_au": dt / inner,
                                 "inner_steps_per_s": ws * inner * 1e3 / ms} if use_respa else None,
                       "chains": "4 links on every coordinate, 3 Yoshida stages", "pme_grid": spec.grid,
                       "plain_force_evaluation_ms": float(np.mean(force_ms)),
                       **({} if use_respa else {
                           "bead_force_evals_per_s": ws * P * 1e3 / ms, "force_ms_per_step": float(np.mean(force_ms)),
                           "pimd_bookkeeping_ms_per_step": ms - float(np.mean(force_ms))}),
                       "list_rebuilds_incl_warmup": rebuilds,
                       "step_ms_median": float(np.median(ms_list)), "step_ms_max": float(np.max(ms_list)),
                       "energies_last_step": {k: e[k] for k in ("vintert", "vintrat", "kin_harm", "akvirx")},
                       "l2": "256 MiB buffer written between timed steps; CUDA events on the launch stream"},
            "roofline": {"bound": "hbm", "kernel": "normal-mode transform (positions -> modes, all beads)",
                         "achieved": t_bytes / (t_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                         "frac": t_bytes / (t_ms * 1e-3) / 1e9 / hbm, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": t_bytes, "ms": t_ms},
            "cpu_baseline": None, "e2e": None, "gpu_launches": None, "clocks": clocks,
        }
        print(json.dumps(line))
    pm.close()
    box.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_respa(args, ws, rank, local):
    """The force calls of one PINY RESPA step on the device: 4096 q-TIP4P/F
    x 32 beads, respa_steps_lrf 2, respa_steps_intra 2 (inner cutoff 5 A,
    switch width 1 A), so int_NVT_pimd's loops ask for the levels
    [innermost, inner inter, innermost, outer] (piny_b200.respa.loop_levels).
    A step is those four calls; the plain evaluation, which a run without
    RESPA makes at each of the four inner time steps, is timed beside it."""
    import dataclasses

    import torch

    from piny_b200 import respa as R
    from piny_b200 import system, water
    from piny_b200.lib import DeviceBox

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    spec = water.named_spec("tip4pf_4096_p32")
    if ws > 1:
        spec = dataclasses.replace(spec, seed=spec.seed + rank)
    pos = water.build_positions(spec) / water.BOHR
    S = system.build_system(spec, pos)
    P = spec.nbeads
    xmod = pos.mean(axis=0)
    box = DeviceBox(S, P, args.precision)
    box.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
    nres = (2, 1, 2, 1)
    rk = {"lrf": nres[0], "intra": nres[2], "pimd": nres[3], "rheal": 1.0, "eq_res": 0.0}
    cut_res = np.minimum(np.asarray(S["cutoff"]), 5.0 / water.BOHR)
    rs = R.respa_setup(*nres, True, True, cut_res, 1.0 / water.BOHR, np.asarray(S["bond_eq"]))
    box.set_respa(rs)
    levels = [lv for lv in R.loop_levels(*nres, True) if lv]
    stream = torch.cuda.current_stream(dev)
    d_pos = torch.from_numpy(pos).to(dev)
    d_xm = torch.from_numpy(xmod).to(dev)
    d_f = torch.empty_like(d_pos)
    d_ft = torch.empty_like(d_pos)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def call(lv):
        box.respa_force_device(d_pos.data_ptr(), d_xm.data_ptr(), S["hmat"], lv, d_f.data_ptr(),
                               d_ft.data_ptr() if lv & R.FULL_INTER else None, stream=stream.cuda_stream,
                               distribute_ghosts=True)

    def timed(fn):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(max(3, args.warmup)):
        for lv in levels:
            call(lv)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if ws > 1:
        torch.distributed.barrier()
    per_level = {lv: [] for lv in set(levels)}
    steps = []
    for _ in range(args.steps):
        tot = 0.0
        for lv in levels:
            t = timed(lambda: call(lv))
            per_level[lv].append(t)
            tot += t
        steps.append(tot)
    plain = [timed(lambda: box.energy_force_device(d_pos.data_ptr(), d_xm.data_ptr(), S["hmat"], d_f.data_ptr(),
                                                   stream=stream.cuda_stream, distribute_ghosts=True))
             for _ in range(max(3, args.steps))]
    clocks = sampler.stop()
    ms = float(np.mean(steps))
    if ws > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    names = {R.RES_INTRA: "innermost (bonds, bends)", R.RES_INTER | R.FULL_INTRA | R.RES_INTRA:
             "inner inter (pairs inside 5 A, bonds, bends)", R.FULL_INTER | R.RES_INTER | R.FULL_INTRA | R.RES_INTRA:
             "outer (everything, weighted and plain)"}
    if rank == 0:
        plain_ms = float(np.mean(plain))
        cpu = None
        if not args.no_cpu_baseline and ws == 1:
            cpu = respa_cpu_baseline(spec, pos * water.BOHR, rk, levels)
        line = {
            "metric": "RESPA steps/s (force calls of one PINY step, TIP4P/F 4096 mol x 32 beads)",
            "value": ws * 1e3 / ms, "unit": "RESPA steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64acc" if args.precision == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": "respa", "molecules": spec.nmol, "beads": P, "respa_steps_lrf": nres[0],
                       "respa_steps_intra": nres[2], "cutoff_res_A": 5.0, "rheal_A": 1.0,
                       "calls_per_step": len(levels),
                       "ms_per_level": {names[lv]: float(np.mean(v)) for lv, v in per_level.items()},
                       "plain_evaluation_ms": plain_ms,
                       "plain_ms_for_the_same_inner_steps": plain_ms * len(levels),
                       "l2": "256 MiB buffer written before each timed call; CUDA events on the launch stream"},
            "roofline": None, "cpu_baseline": cpu, "e2e": None, "gpu_launches": None, "clocks": clocks,
        }
        print(json.dumps(line))
    box.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def respa_cpu_baseline(spec, pos_A, rk, levels):
    """PINY's own CPU path (oracle/_ref/piny_ref respa_time) on the same box
    with the same RESPA input: each level once on 2 of the beads, 1 core,
    after one warm-up round; one RESPA step = the step's levels, scaled to
    all beads."""
    from piny_b200 import respa as R
    from piny_b200 import water
    exe = piny_ref_binary()
    if not exe:
        return None
    d = tempfile.mkdtemp(prefix="piny_respa_")
    water.write_piny_input(d, spec, pos_A, respa=rk)
    r = subprocess.run([exe, "respa_time", d, "water.input", "1", "2"], capture_output=True, text=True)
    shutil.rmtree(d, ignore_errors=True)
    if r.returncode != 0:
        return None
    t = {int(l.split()[1]): float(l.split()[2]) for l in r.stdout.splitlines() if l.startswith("level")}
    # piny_ref's level order: outer, inner inter, full intra, innermost
    code = {R.FULL_INTER | R.RES_INTER | R.FULL_INTRA | R.RES_INTRA: 0, R.RES_INTER | R.FULL_INTRA | R.RES_INTRA: 1,
            R.FULL_INTRA | R.RES_INTRA: 2, R.RES_INTRA: 3}
    step_s = sum(t[code[lv]] for lv in levels) * spec.nbeads / 2.0
    return {"value": 1.0 / step_s, "unit": "RESPA steps/s", "cores": 1, "kind": "reference",
            "sample": "PINY's energy_control sub-steps at each RESPA level (oracle/_ref/piny_ref respa_time), "
                      "2 of 32 beads per level, 1 host core, after one warm-up round; scaled to 32 beads",
            "seconds_per_level_2_beads": {str(k): v for k, v in t.items()}}


def run_batch(args, ws, rank, local):
    """64 uneven TIP4P/F boxes, all beads, one CUDA graph launch per step:
    the faster (timed at capture) of the multi-box kernels (one persistent
    launch per phase and shape group) and one graph branch per box, unless
    --batch-kernels or --batch-branches pins one."""
    import torch

    from piny_b200 import system, water
    from piny_b200.lib import DeviceBatch, DeviceBox

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    nbox = int(args.config[len("c4_batch"):] or 64)
    specs = water.c4_specs(nbox=nbox, seed=2024 + 1000 * rank)
    boxes, keep, d_pos, d_xm, d_f, hm, pins = [], [], [], [], [], [], []
    alg = 0.0
    t0 = time.perf_counter()
    for sp in specs:
        pos = water.build_positions(sp) / water.BOHR
        S = system.build_system(sp, pos)
        b = DeviceBox(S, sp.nbeads, args.precision)
        xmod = pos.mean(axis=0) if sp.nbeads > 1 else None
        npairs = b.build_list(pos[0], xmod, S["hmat"], S["cutskin2"])
        d = torch.from_numpy(pos).to(dev)
        dx = torch.from_numpy(xmod).to(dev) if xmod is not None else None
        f = torch.empty_like(d)
        keep += [d, dx, f]
        pins.append((torch.from_numpy(pos.copy()).pin_memory(), torch.empty(pos.shape, dtype=torch.float64).pin_memory()))
        boxes.append(b)
        d_pos.append(d.data_ptr())
        d_xm.append(None if dx is None else dx.data_ptr())
        d_f.append(f.data_ptr())
        hm.append(S["hmat"])
        alg += sp.nbeads * alg_bytes_per_bead_eval(S, sp.nbeads, npairs, args.precision)
    setup_s = time.perf_counter() - t0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch = DeviceBatch(boxes)
    stream = torch.cuda.current_stream(dev)
    tune_ms, tune_keep = batch.tune(d_pos, d_xm, hm, d_f, stream=stream.cuda_stream)
    choices = [b.tuning() for b in boxes]
    tune_s = time.perf_counter() - t0
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    br, bk = args.batch_branches, args.batch_kernels
    for _ in range(max(3, args.warmup)):
        batch.energy_force_device(d_pos, d_xm, hm, d_f, stream=stream.cuda_stream, branches=br, kernels=bk)
    torch.cuda.synchronize()
    fused, graph_launches = batch.last_mode()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    step_ms = []
    for _ in range(args.steps):
        flush.zero_()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        batch.energy_force_device(d_pos, d_xm, hm, d_f, stream=stream.cuda_stream, branches=br, kernels=bk)
        ev1.record(stream)
        ev1.synchronize()
        step_ms.append(ev0.elapsed_time(ev1))
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    clocks = sampler.stop()
    ms = float(np.mean(step_ms))
    if ws > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    nbead = sum(sp.nbeads for sp in specs)
    value = ws * nbead / (ms * 1e-3)
    # end to end: positions from pinned host memory in, forces out, every step
    e2e_ms = []
    for k in range(args.steps + 2):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for i in range(nbox):
            keep[3 * i].copy_(pins[i][0], non_blocking=True)
        batch.energy_force_device(d_pos, d_xm, hm, d_f, stream=stream.cuda_stream, branches=br, kernels=bk)
        for i in range(nbox):
            pins[i][1].copy_(keep[3 * i + 2], non_blocking=True)
        ev1.record(stream)
        ev1.synchronize()
        if k >= 2:
            e2e_ms.append(ev0.elapsed_time(ev1))
    e2e = float(np.mean(e2e_ms))
    # each form pinned, for the record (the timed steps above ran the kept one)
    forms_ms = {}
    for name, fb, fk in (("multi_box_kernels", False, True), ("branches", True, False)):
        ts = []
        for k in range(6):
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            batch.energy_force_device(d_pos, d_xm, hm, d_f, stream=stream.cuda_stream, branches=fb, kernels=fk)
            ev1.record(stream)
            ev1.synchronize()
            if k >= 1:
                ts.append(ev0.elapsed_time(ev1))
        forms_ms[name] = {"ms": float(np.median(ts)), "launches": batch.last_mode()[1]}
    if args.profile_step:
        # one more step of the kept (or pinned) form between cudaProfilerStart
        # and Stop, for `ncu --profile-from-start off` launch lists
        batch.energy_force_device(d_pos, d_xm, hm, d_f, stream=stream.cuda_stream, branches=br, kernels=bk)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        batch.energy_force_device(d_pos, d_xm, hm, d_f, stream=stream.cuda_stream, branches=br, kernels=bk)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    hbm, peak_kind = peaks()
    achieved = alg / (ms * 1e-3) / 1e9
    nbytes = sum(int(p[0].numel()) * 8 for p in pins)
    c4_cpu = None
    if rank == 0 and not args.no_cpu_baseline and piny_ref_binary():
        try:
            t = piny_bead_seconds(specs, reps=3)
            c4_cpu = {"value": float(nbead / np.sum([sp.nbeads * t[i] for i, sp in enumerate(specs)])),
                      "unit": UNIT, "cores": 1, "kind": "reference",
                      "sample": "PINY (oracle/_ref/piny_ref): 1 bead of each of the %d boxes, median of 3 after "
                                "a warm-up (boxes run as concurrent single-threaded processes); a step = every "
                                "bead of every box on one core" % nbox, **cpu_info()}
        except Exception as exc:  # reported, not fatal
            c4_cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": "failed: %s" % exc}
    if rank == 0:
        line = {
            "metric": "bead-force evals/s (64 uneven TIP4P/F boxes, batched)", "value": value, "unit": UNIT,
            "n_gpus": ws, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64acc" if args.precision == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": args.config, "boxes": nbox, "bead_evals_per_step": nbead,
                       "molecules": [sp.nmol for sp in specs], "beads": [sp.nbeads for sp in specs],
                       "pme_grid": [sp.grid for sp in specs], "precision": args.precision,
                       "tuning": choices, "tuning_set": {"kept": tune_keep, "batch_ms": tune_ms},
                       "setup_s": setup_s, "autotune_s": tune_s,
                       "l2": "256 MiB buffer written between timed steps; CUDA events on the launch stream",
                       "launch": ("one CUDA graph launch per step: multi-box kernels, one persistent launch "
                                  "per phase and shape group (%d kernel nodes for %d boxes)" % (graph_launches, nbox))
                       if fused else ("one CUDA graph launch per step (boxes as parallel branches, "
                                      "%d kernel nodes)" % graph_launches),
                       "forms_ms": forms_ms},
            "roofline": {"bound": "hbm", "kernel": "whole batch step", "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg,
                         "bytes_model": "per bead-eval 48 B/site + 4 B x list/P + 6 grid passes"},
            "cpu_baseline": c4_cpu,
            "e2e": {"value": ws * nbead / (e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "ms_per_step": e2e},
            "gpu_launches": graph_launches * args.steps,
            "clocks": clocks,
        }
        print(json.dumps(line))
    batch.close()
    for b in boxes:
        b.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------

def main():
    args = parse_args()
    ws, rank, local = dist_init()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    if args.config.startswith("c4_batch"):
        return run_batch(args, ws, rank, local)
    if args.config == "c5_grad":
        return run_grad(args, ws, rank, local)
    if args.config in ("pimd_nvt", "pimd_nvt_respa"):
        return run_pimd(args, ws, rank, local)
    if args.config == "respa":
        return run_respa(args, ws, rank, local)
    if args.config.startswith("list_"):
        return run_list(args, ws, rank, local)

    import torch

    from piny_b200 import system, water
    from piny_b200.lib import DeviceBox

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    spec = water.named_spec(args.config)
    if ws > 1:
        spec.seed = spec.seed + rank
    pos_A = water.build_positions(spec)
    pos = pos_A / water.BOHR
    S = system.build_system(spec, pos)
    xmod = pos.mean(axis=0)
    P = spec.nbeads
    natm = S["natm"]
    hmat = S["hmat"]

    box = DeviceBox(S, P, args.precision)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    npairs = box.build_list(pos[0], xmod, hmat, S["cutskin2"])
    list_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream(dev)
    d_pos = torch.from_numpy(pos).to(dev)
    d_xmod = torch.from_numpy(xmod).to(dev)
    d_force = torch.empty_like(d_pos)
    # launch shapes: pinned by --tuning, else the project's autotuner on these inputs
    tuning = {}
    if args.tuning:
        box.set_tuning([int(v) for v in args.tuning.split(",")])
        tuning[args.precision] = box.tuning()
    else:
        tuning[args.precision] = box.autotune(d_pos.data_ptr(), d_xmod.data_ptr(), hmat, reps=3,
                                              energy=not args.no_energy)[0]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step(b, force):
        return b.energy_force_device(d_pos.data_ptr(), d_xmod.data_ptr(), hmat, force.data_ptr(),
                                     stream=stream.cuda_stream, energy=not args.no_energy)

    for _ in range(max(3, args.warmup)):
        step(box, d_force)
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    step_ms, phase = [], np.zeros(4)
    for _ in range(args.steps):
        flush.zero_()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        step(box, d_force)
        ev1.record(stream)
        ev1.synchronize()
        step_ms.append(ev0.elapsed_time(ev1))
        phase += np.array(box.last_timing()[:4])
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    clocks = sampler.stop()
    ms = float(np.mean(step_ms))
    if ws > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = ws * P / (ms * 1e-3)
    phase /= args.steps
    force_mixed = d_force.cpu().numpy()

    # FP64 device path on the same box (the comparison the metric names)
    fp64 = None
    if not args.no_fp64:
        box64 = DeviceBox(S, P, "fp64")
        box64.build_list(pos[0], xmod, hmat, S["cutskin2"])
        if not args.tuning:
            tuning["fp64"] = box64.autotune(d_pos.data_ptr(), d_xmod.data_ptr(), hmat, reps=3,
                                            energy=not args.no_energy)[0]
        f64 = torch.empty_like(d_pos)
        for _ in range(2):
            step(box64, f64)
        t64 = []
        nrep = max(2, min(args.steps, 5))
        for _ in range(nrep):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step(box64, f64)
            e1.record(stream)
            e1.synchronize()
            t64.append(e0.elapsed_time(e1))
        f64n = f64.cpu().numpy()
        err = float(np.linalg.norm(force_mixed - f64n) / np.linalg.norm(f64n))
        ms64 = float(np.mean(t64))
        fp64 = {"value": ws * P / (ms64 * 1e-3), "ms_per_step": ms64, "force_rel_rms_mixed_vs_fp64": err}
        box64.close()

    # end to end through the public host-buffer call (pinned host memory)
    pin_pos = torch.from_numpy(pos.copy()).pin_memory()
    pin_xm = torch.from_numpy(xmod.copy()).pin_memory()
    pin_f = torch.empty_like(pin_pos).pin_memory()
    from piny_b200.lib import PinyEnergies, _pd
    import ctypes as C
    hm = np.ascontiguousarray(hmat)
    e2e_ms = []
    for k in range(args.steps + 2):
        e = PinyEnergies()
        rc = box.L.pinyb200_energy_force(box.h, C.cast(C.c_void_p(pin_pos.data_ptr()), _pd),
                                         C.cast(C.c_void_p(pin_xm.data_ptr()), _pd), hm.ctypes.data_as(_pd), 0,
                                         C.cast(C.c_void_p(pin_f.data_ptr()), _pd), C.byref(e))
        assert rc == 0, box.L.pinyb200_last_error(box.h)
        if k >= 2:
            e2e_ms.append(box.last_timing()[4])
    e2e = float(np.mean(e2e_ms))
    if ws > 1:
        t = torch.tensor([e2e], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e = float(t.item())
    h2d = pos.nbytes + xmod.nbytes
    d2h = pos.nbytes + C.sizeof(PinyEnergies)

    # every kernel serialised (events after each), with its HBM fraction
    linfo = box.list_info()
    kernels = kernel_profile(box, lambda: step(box, d_force), S, P, args.precision, npairs,
                             linfo.get("nmol_pairs", 0), flush, stream)
    # roofline of the dominant kernel by serialised time; its duration is
    # the one measured inside the timed steps (pair phase events / PME phase)
    hbm, peak_kind = peaks()
    names = ["total", "pair", "pme", "intra"]
    dom_k = max(kernels, key=lambda k: k["ms"])
    pme_ms = sum(k["ms"] for k in kernels if k["kernel"].startswith("pme_"))
    if dom_k["kernel"] == "pair" or dom_k["ms"] >= pme_ms:
        # the scope table's per bead-eval figure for the pair kernel:
        # 48 B/site (FP64 positions in, forces out) + 4 B x list pairs / P
        alg_bytes = 48.0 * natm * P + 4.0 * npairs
        dom_name, dom_ms = "pair", float(phase[1])
        unit_note = "48 B/site/bead (FP64 positions + forces) + 4 B per Verlet-list pair per launch"
    else:
        G = S["ngrid_a"] * S["ngrid_b"] * S["ngrid_c"]
        bg = 8 if args.precision == "mixed" else 16
        alg_bytes = P * 6.0 * G * bg
        dom_name, dom_ms = "pme phase", float(phase[2])
        unit_note = "per bead 6 grid passes x %d B/point" % bg
    achieved = alg_bytes / (dom_ms * 1e-3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        try:
            traffic = json.load(open(tf)).get("%s_%s_%s" % (args.config, args.precision, dom_name.split()[0]))
        except Exception:
            traffic = None
    roof = {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": alg_bytes, "bytes_model": unit_note,
            "duration_ms": dom_ms, "duration_from": "pair-phase CUDA events of the timed steps (PME concurrent)"
            if dom_name == "pair" else "PME-phase CUDA events of the timed steps",
            "phase_ms": {names[i]: float(phase[i]) for i in range(4)}}

    # against PINY itself: forces of the beads PINY's evaluation of this
    # box stored (tests/golden), device run on the positions PINY used
    piny = None
    gold = piny_golden(args.config)
    if gold is not None:
        F, gpos, gxm = gold
        piny = {"beads": [int(b) for b in F["ref_beads"]], "npairs_piny": int(F["npairs"])}
        for prec in ("mixed", "fp64"):
            bx = DeviceBox(S, P, prec)
            bx.build_list(gpos[0], gxm, F["hmat"], F["cutskin2"])
            fg, eg = bx.energy_force(gpos, gxm, F["hmat"])
            ref = F["ref_force_raw"]
            piny["force_rel_rms_%s" % prec] = float(np.linalg.norm(fg[F["ref_beads"]] - ref) / np.linalg.norm(ref))
            piny["vintert_rel_%s" % prec] = float(abs(eg["vintert"] - F["ref_vintert"]) / abs(F["ref_vintert"]))
            piny["npairs_%s" % prec] = int(bx.list_info()["npairs"])
            bx.close()
    # the bound that applies to the pair kernel: FP32 issue, not HBM
    alu = None
    try:
        from piny_b200.lib import fma_peak_gflops
        npc = in_cutoff_pairs(box, S, pos[0], xmod)
        flops = 40.0 * npc * P
        peak32 = fma_peak_gflops(fp64=args.precision == "fp64")
        ach = flops / (phase[1] * 1e-3) / 1e9
        alu = {"bound": "fp32" if args.precision == "mixed" else "fp64", "kernel": "pair phase",
               "achieved": ach, "peak": peak32, "unit": "GFLOP/s", "frac": ach / peak32, "peak_kind": "measured",
               "flops_per_launch": flops, "in_cutoff_site_pairs": int(npc),
               "flops_model": "40 flops per in-cutoff site pair and bead (bead-1 pair count x beads)"}
    except Exception as exc:  # reported, not fatal
        alu = {"error": str(exc)}

    # Verlet-list builds of this box (host call and device rebuild)
    try:
        lists = list_timing(S, P, spec.model.nsite, pos, xmod, args.precision, dev, reps=3)
    except Exception as exc:  # reported, not fatal
        lists = {"error": str(exc)}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(spec, pos_A, pos, S, xmod)
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": "failed: %s" % exc}

    if rank == 0:
        line = {
            "metric": metric_for(args.config, spec), "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64acc" if args.precision == "mixed" else "f64",
            "data": "synthetic",
            "config": box_config(spec, args, int(natm), int(S["ngrid_a"]), int(npairs), list_s),
            "tuning": {k: {"pme_tile": v[0], "pair_kernel": v[1], "pair_blocks_per_sm": v[2], "pme_overlap": v[3]}
                       for k, v in tuning.items()},
            "roofline": roof,
            "kernels": kernels,
            "vs_piny": piny,
            "alu_roofline": alu,
            "list_build": lists,
            "cpu_baseline": cpu,
            "e2e": {"value": ws * P / (e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e},
            "fp64_gpu": fp64,
            "speedup_vs_fp64_gpu": (value / fp64["value"]) if fp64 else None,
            "gpu_launches": box_launches(S, P) * args.steps,
            "clocks": clocks,
        }
        print(json.dumps(line))
    box.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def in_cutoff_pairs(box, S, pos1, xmod):
    """Force-bearing site pairs of the list within their cutoff on bead 1
    (minimum image through the mode-1 positions, as the kernels take it)."""
    pi, pj = box.get_list()
    q = S["charge"]
    typ = S["atm_typ"]
    ntyp = S["ntyp"]
    a, b = np.minimum(typ[pi], typ[pj]) + 1, np.maximum(typ[pi], typ[pj]) + 1
    pt = ((a - 1) * ((ntyp + 1) * 2 - a)) // 2 + b - a
    u = S["inter_map"][pt]
    nspl = S["nsplin"]
    has_vdw = np.array([np.any(S["cdv0"][k * nspl:(k + 1) * nspl] != 0) for k in range(S["ninter_unique"])])
    act = (q[pi] * q[pj] != 0) | has_vdw[u]
    pi, pj, pt = pi[act], pj[act], pt[act]
    h = np.asarray(S["hmat"]).reshape(3, 3, order="F")
    hi = np.linalg.inv(h)
    d = pos1[pi] - pos1[pj]
    if xmod is not None:
        dm = xmod[pi] - xmod[pj]
        d -= (h @ np.round(hi @ dm.T)).T
    else:
        d -= (h @ np.round(hi @ d.T)).T
    r = np.sqrt((d * d).sum(1))
    return int(np.count_nonzero(r < S["cutoff"][pt]))


def box_launches(S, P):
    """Kernels one evaluation launches (memsets are not kernels): transpose
    in, ghost positions, the pair kernel, PME (bin, spread, plane FFT,
    c-axis FFT with the convolution, inverse plane FFT, gather), bond, bend,
    excluded-pair correction, transpose out."""
    n = 1 + (1 if S.get("nghost", 0) else 0) + 1
    if int(np.count_nonzero(S["charge"])) and S.get("nktot", 0):
        n += 6
    n += (1 if S.get("nbond", 0) else 0) + (1 if S.get("nbend", 0) else 0) + (1 if S.get("necor", 0) else 0)
    return n + 1


if __name__ == "__main__":
    sys.exit(main())
