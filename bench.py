#!/usr/bin/env python
"""Benchmark: time-to-converged-labels of EGG-SynC on one B200.

Workload: 1,000,000 x 3 points, 50 Gaussian clusters (centres U[0.1,0.9]^3,
per-cluster std U[0.005,0.03]), 10% uniform noise, min-max normalised,
eps = 0.015 (eggsync.data.c5, seed 0).  One step = one full EGG-SynC run
from positions to converged labels.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* value: seconds per run with the input already in HBM and the labels left
  in HBM (device buffers through the C ABI), CUDA events on the calling
  stream, L2 flushed (256 MiB write) before every timed step.
* e2e: the same through the public API with pinned host buffers: the
  host-to-device copy of the points and the device-to-host copy of the labels
  are inside every timed step.
* roofline: the update kernel (the dominant kernel), timed with CUDA events
  on its launching stream in a profiled run.
* cpu_baseline: the reference's own CPU SynC (src/algorithms/SynC.cpp, built
  from its sources into oracle/_ref) on a bounded sample of the same workload.
* learned (N = 1): the same workload with the learned warm start
  (eggsync/models/warm_d3.npz, unverified): time, iterations and the
  adjusted Rand index of its partition against the plain run's.
* batched_sweep (N = 1): 64 datasets x 8 eps (512 runs) in one batched call
  against 512 sequential calls, with an identity check of all labels.
  --no-extra skips these two legs.

With --gpus N (under torchrun) every rank runs its own replica (the loop does
not shard); value is the max over ranks.  --impl reference times the
reference's CPU SynC on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from datetime import timedelta
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "egg-sync_b200"))

METRIC = "time-to-converged-labels (s) at 1M x 3D"
WORKLOAD = "egg-sync plain loop, 1M x 3D, 50 Gaussian clusters + 10% noise, eps 0.015 (c5 shape, seed 0)"
L2_FLUSH_BYTES = 256 << 20
# Iterations the reference CPU SynC takes on this workload: its lambda stop
# rule (SynC.cpp:277) reached after 10 iterations, r_local 0.99933, counted
# by `python bench.py --sync-iterations` (the brute-force GPU SynC follows
# the same rule; 15 s on one B200).  Used only to extrapolate the CPU
# baseline, whose full run would take hours.
C5_SYNC_ITERATIONS = 10
# points in the timed sample of the CPU baseline
CPU_SAMPLE = 4000
# DRAM bytes (read + written) of one update launch on this workload: the mean
# of iterations 2-4 (72.1 MB read + 4.8 MB written), from a bounded ncu capture
# of the dram__bytes counters (ncu -k regex:k_update -s 193 -c 3 on
# python bench.py --profile-run; cold cache: ncu flushes between replays).
UPDATE_DRAM_BYTES_PER_LAUNCH = 76.9e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-extra", action="store_true", help="skip the learned and batched-sweep legs")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--cpu-sample", type=int, default=0, help="points in the CPU-baseline sample (0 = auto)")
    ap.add_argument("--profile-run", action="store_true",
                    help="for ncu: one warm-up run and one run of the workload through the host-driven loop, "
                         "no timing, no CPU baseline")
    ap.add_argument("--sync-iterations", action="store_true",
                    help="count the reference CPU SynC's iterations on the workload (brute-force GPU SynC)")
    ap.add_argument("--sync-max-iter", type=int, default=300)
    ap.add_argument("--profile-warm", action="store_true",
                    help="for ncu: one warm-up run and one warm-started run of the workload (learned "
                         "warm start), no timing")
    ap.add_argument("--stage-split", action="store_true",
                    help="per-phase split of the loop graph's time (iterations 0-11, 12-59, 60+) from the "
                         "per-iteration %%globaltimer stamps, and the slowest iterations")
    ap.add_argument("--profile-grid", action="store_true",
                    help="for ncu: six grid builds of the workload from device-resident points (L2 flushed "
                         "before each), no timing")
    return ap.parse_args()


def profile_run(args):
    """One warm-up run and one run (host-driven loop: plain kernel launches)."""
    import torch

    from eggsync import data, egg_sync

    dev = torch.device("cuda", 0)
    c = data.c5(args.seed, n=args.n)
    Xd = torch.from_numpy(c["X"]).to(dev)
    lab = torch.empty(len(c["X"]), dtype=torch.int32, device=dev)
    for k in range(2):
        _, info = egg_sync(Xd, c["eps"], labels_out=lab, loop="host")
    torch.cuda.synchronize(dev)
    print(json.dumps({"profile_run": True, "n": len(c["X"]), "iterations": info["iterations"],
                      "launches_per_run": info["launches"]}))


def profile_warm(args):
    """One warm-up run and one run with the learned warm start (features,
    tensor-core inference, displacement, then the plain loop)."""
    import torch

    from eggsync import data, egg_sync, warm

    dev = torch.device("cuda", 0)
    c = data.c5(args.seed, n=args.n)
    Xd = torch.from_numpy(c["X"]).to(dev)
    lab = torch.empty(len(c["X"]), dtype=torch.int32, device=dev)
    model = warm.default_model(3)
    for k in range(2):
        _, info = egg_sync(Xd, c["eps"], labels_out=lab, warm_start=model)
    torch.cuda.synchronize(dev)
    print(json.dumps({"profile_warm": True, "n": len(c["X"]), "iterations": info["iterations"],
                      "warm_ms": info["warm_ms"]}))


def stage_split(args):
    """Where the loop graph's time goes by phase of the run, on the device's
    own clock: each iteration stamps its start, the update's start, the end
    of the update (the extra-check gate) and its end; runs stopped after 12
    and 60 iterations follow the full run's trajectory exactly, so the
    differences of the stage sums give each phase (median of 4 runs each)."""
    import numpy as np
    import torch

    from eggsync import data, egg_sync

    dev = torch.device("cuda", 0)
    c = data.c5(args.seed, n=args.n)
    Xd = torch.from_numpy(c["X"]).to(dev)
    lab = torch.empty(len(c["X"]), dtype=torch.int32, device=dev)

    def runs(k):
        rows, info = [], None
        for r in range(5):
            _, info = egg_sync(Xd, c["eps"], labels_out=lab, max_iter=k)
            rows.append(info["stage_ms"][1:4] + [info["grid_builds"], info["extra_checks"], info["total_ms"]])
        return np.median(np.array(rows[1:]), 0), info

    s12, _ = runs(12)
    s60, _ = runs(60)
    sall, info = runs(0)
    iters = info["iterations"]
    out = {"workload": "1M x 3D (c5 shape), eps %.3f" % c["eps"], "iterations": iters, "total_ms": sall[5],
           "columns": ["before the update (grid check, sort, cell sums, need)", "update",
                       "update end to iteration end (extra check when it runs)"]}
    for name, hi, lo, n_it in (("0-11", s12, None, 12), ("12-59", s60, s12, 48), ("60+", sall, s60, iters - 60)):
        dlt = hi if lo is None else hi - lo
        out[name] = {"ms": [round(float(v), 3) for v in dlt[:3]], "us_per_iteration": [
            round(float(v) * 1e3 / n_it, 1) for v in dlt[:3]], "grid_builds": int(dlt[3]), "extra_checks": int(dlt[4])}
    itr = np.array(info["itr_ms"])
    top = np.argsort(-itr)[:5]
    out["slowest_iterations_ms"] = {int(k): round(float(itr[k]), 3) for k in top}
    print(json.dumps(out))


def profile_grid(args):
    """Six builds of the double grid (egg_sync_grid) of the workload from
    device-resident points, the L2 flushed before each: every grid/scan kernel
    runs on a fresh input (no unchanged-grid early exit)."""
    import torch

    from eggsync import data, egg_grid

    dev = torch.device("cuda", 0)
    c = data.c5(args.seed, n=args.n)
    Xd = torch.from_numpy(c["X"]).to(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    for _ in range(6):
        flush.zero_()
        _, _, start = egg_grid(Xd, c["eps"])
    torch.cuda.synchronize(dev)
    print(json.dumps({"profile_grid": True, "n": len(c["X"]), "cells": len(start) - 1}))


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() and args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
        pg = dist
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return rank, local, world, pg


def max_over_ranks(pg, vals, device):
    """Each value's maximum over the ranks (an all-reduce MAX); the values
    themselves with one rank.  Every rank gets the result."""
    if pg is None:
        return [float(v) for v in vals]
    import torch

    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path("/tmp/egg_bench_clocks_%d.csv" % os.getpid())

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        try:
            self.path.unlink()
        except Exception:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def update_bytes_per_launch(n, d, cells):
    """Algorithmic bytes of one update launch: read each point's position and
    its (sin, 1-cos) offsets once, read each cell's record (start, dims, two
    sums) once, write each point's new position."""
    return n * (4 * d + 8 * d + 4 * d) + cells * (4 + 4 * d + 8 * d)


def grid_bytes(n, d, width, cells, n_outer):
    """Algorithmic bytes of one full grid build from device-resident points
    (egg_sync_grid, the grid of EGG_SynC.cu:248-341): the input transpose
    (row-major read, per-dimension write, original index), the grid check's
    copy, the radix sort, the tile histograms, the gather into sorted
    order, the cell heads and records, the outer ranges.  The sort: for
    d <= 3 with at most 256 cells per dimension one 32-bit key per point is
    computed once (d coordinates read, key and position written) and 1 + d
    passes each read the keys for the histogram and move (key, position)
    pairs (the last pass writes positions only); otherwise each pass reads
    its digit through the permutation (all d coordinates in the first,
    sub-cell pass) and reads and writes the permutation."""
    tiles = (n + 2047) // 2048                # 2048-point tiles
    per_point = (4 * d + 4 * d + 4)          # transpose
    per_point += 8 * d                       # grid check: read Xn, write X
    if d <= 3 and width <= 256:
        passes = 1 + d
        per_point += 4 * d + 8               # keys: coordinates in; key, position out
        per_point += passes * (4 + 16) - 4   # per pass: hist (key), scatter (key, position in and out)
    else:
        digits = 1 if width <= 256 else 2
        passes = 1 + d * digits
        per_point += 4 * d + 4 * d + 4       # sub-cell pass: hist + scatter (first pass reads no permutation)
        per_point += (passes - 1) * (8 + 12)  # later passes: hist (perm + digit), scatter (perm + digit + perm out)
    per_point += 4 + 4 * d + 4 + 4 * d + 4   # gather: perm, Xn, orig in; X, orig_tmp out
    per_point += 4 * d + 4 + 4 + 4           # heads: X, orig_tmp in; cell_of, orig out
    hist = passes * tiles * 256 * 4 * 4      # histogram write, scan read + write, scatter read
    return n * per_point + cells * (4 + 4 * d + 4 + 8) + (n_outer + 1) * 12 + hist


def grid_leg(Xd, eps, dev, flush, reps=10):
    """The grid build (egg_sync_grid, device input and outputs) timed with
    CUDA events on the calling stream, the L2 flushed before each build;
    against the measured HBM bandwidth."""
    import torch

    from eggsync import egg_grid

    n, d = Xd.shape
    out = (torch.empty(n, dtype=torch.int32, device=dev), torch.empty(n, dtype=torch.int32, device=dev),
           torch.empty(n + 1, dtype=torch.int32, device=dev))
    stream = torch.cuda.current_stream(dev)
    for _ in range(3):
        _, _, start = egg_grid(Xd, eps, out=out)
    times = []
    for _ in range(reps):
        flush.zero_()
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        _, _, start = egg_grid(Xd, eps, out=out)
        e.record(stream)
        e.synchronize()
        times.append(s.elapsed_time(e))
    ms = statistics.median(times)
    side = float(np.float32(np.sqrt((eps / 2) ** 2 / d)))
    width = int(np.float32(1.0) / np.float32(side))
    od = min(d, int(np.log(n) / np.log(width)))
    b = grid_bytes(n, d, width, len(start) - 1, width ** od)
    peak, kind = measured_peaks()
    ach = b / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": "grid build (egg_sync_grid: transpose, check, radix passes, heads, outer ranges)",
            "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_source": kind,
            "ms_per_build": ms, "algorithmic_bytes": b, "cells": len(start) - 1,
            "note": "the timed call includes the entry point's two host synchronisations and its output copies "
                    "(order, cell_of, cell_start); per-kernel DRAM bytes and times: profiles/grid_scan_c5_1M.md"}


_STATS_CHILD = r"""
import ctypes as C, json, os, sys
sys.path.insert(0, sys.argv[1])
from eggsync import _lib, data, egg_sync
c = data.c5(int(sys.argv[2]), n=int(sys.argv[3]))
egg_sync(c["X"], c["eps"])
out = (C.c_int64 * 64)()
k = _lib.load().egg_update_counters(out, 64)
print(json.dumps(dict(zip(_lib.UPDATE_COUNTERS, [int(v) for v in out[:k]]))))
"""


def update_fp32_leg(args, update_ms):
    """Algorithmic FP32 work of the update kernel over one run, from the
    interaction counters of the stats build (libeggsync_stats.so, same
    results), over the update kernel's CUDA-event time of the profiled run,
    against the nominal FP32 rate of the chip (148 SMs x 128 lanes x 2 flops
    x the measured SM clock).  Flops counted: the reference's box test per
    visited cell (3 per dimension: two fused face offsets and a square), the
    tight-box test per passing cell, 6 per dimension per aggregated cell or
    group (the frame change), 3 per dimension per point-pair distance test
    and 2 per dimension per counted pair."""
    lib = REPO / "egg-sync_b200" / "lib" / "libeggsync_stats.so"
    if not lib.exists():
        return None
    env = dict(os.environ, EGGSYNC_LIB=str(lib))
    r = subprocess.run([sys.executable, "-c", _STATS_CHILD, str(REPO / "egg-sync_b200"), str(args.seed), str(args.n)],
                       env=env, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        return {"error": r.stderr[-500:]}
    k = json.loads(r.stdout.strip().splitlines()[-1])
    d = 3
    flops = (3 * d * k["cells"] + 3 * d * k["small_pass"] +
             6 * d * (k["full"] + k["tight_in"] + k["groups_in"]) + 3 * d * k["pairs"] + 2 * d * k["pairs_in"])
    ach = flops / (update_ms * 1e-3) / 1e12
    peak = 148 * 128 * 2 * 1.965e9 / 1e12
    return {"bound": "fp32", "kernel": "k_update", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
            "frac": ach / peak, "peak_source": "nominal (148 SMs x 128 FP32 lanes x 2 x 1965 MHz)",
            "algorithmic_flops": flops, "counters": k,
            "note": "issue-bound, not FP32-bound: warp-issue and lane-activity figures from ncu in "
                    "profiles/k_update_c5_1M.md"}


def cpu_sample_idx(n, sample):
    """The points whose reference CPU SynC iteration is timed: a fixed random
    sample (seed 0), the same in the cpu_baseline leg and the reference arm."""
    return np.sort(np.random.default_rng(0).choice(n, sample, replace=False)).astype(np.int32)


def cpu_iteration_time(R, X, eps, sample):
    """Seconds of one reference CPU SynC iteration over all n points,
    estimated from `sample` points timed against all n (each point's work is
    one pass over all n points: SynC.cpp:16-56)."""
    idx = cpu_sample_idx(len(X), sample)
    t0 = time.perf_counter()
    R.step_sample(X, eps, idx)
    dt = time.perf_counter() - t0
    return dt / sample * len(X), dt


def cpu_baseline(X, eps, sample, full_c1=True):
    """Reference CPU SynC (SynC.cpp, OpenMP, all host threads): one iteration
    over all n points estimated from a timed sample, times the CPU SynC's own
    iteration count on this workload (an extrapolation: a full run is hours);
    plus one measured full run to labels at 10,000 x 2D (eggsync.data.c1)."""
    sys.path.insert(0, str(REPO / "oracle"))
    from eggsync import data
    from oracle import RefSync

    R = RefSync()
    n = len(X)
    per_iter, dt = cpu_iteration_time(R, X, eps, sample)
    out = {
        "value": per_iter * C5_SYNC_ITERATIONS,
        "unit": "s",
        "cores": R.threads(),
        "kind": "reference",
        "sample": "reference SynC parallel (OpenMP): one iteration of %d sampled points (seed 0) against all %d, "
                  "%.2f s -> %.1f s per full iteration; extrapolated x %d iterations, the CPU SynC's own count on "
                  "this workload (lambda stop rule, counted with the brute-force GPU SynC, bench.py "
                  "--sync-iterations)" % (sample, n, dt, per_iter, C5_SYNC_ITERATIONS),
        "s_per_iteration": per_iter,
        "extrapolated": True,
    }
    if full_c1:
        c = data.c1(0)
        t0 = time.perf_counter()
        _, it = R.run(c["X"], c["eps"], c["lam"])
        out["measured_c1"] = {"workload": "10,000 x 2D, eps 0.05, lambda 1-1e-3 (c1, seed 0)",
                              "time_to_labels_s": time.perf_counter() - t0, "iterations": it}
    return out


def run_ours(args, rank, local, world, pg):
    import torch

    from eggsync import data, egg_sync

    dev = torch.device("cuda", local)
    c = data.c5(args.seed, n=args.n)
    X, eps = c["X"], c["eps"]
    n, d = X.shape
    Xd = torch.from_numpy(X).to(dev)
    lab_d = torch.empty(n, dtype=torch.int32, device=dev)
    Xh = torch.from_numpy(X).pin_memory()
    lab_h = torch.empty(n, dtype=torch.int32).pin_memory()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    for _ in range(max(args.warmup, 0)):
        _, info = egg_sync(Xd, eps, labels_out=lab_d)
    egg_sync(Xh.numpy(), eps, labels_out=lab_h.numpy())

    def barrier():
        if pg is not None:
            pg.barrier()

    def timed(fn):
        times = []
        barrier()
        torch.cuda.synchronize(dev)
        for _ in range(args.steps):
            flush.zero_()
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
            out = fn()
            e.record(stream)
            e.synchronize()
            times.append(s.elapsed_time(e))
        torch.cuda.synchronize(dev)
        barrier()
        return times, out

    with Clocks(local) as clk:
        dev_times, (lab, info) = timed(lambda: egg_sync(Xd, eps, labels_out=lab_d))
    clocks = clk.summary()
    e2e_times, (lab2, info2) = timed(lambda: egg_sync(Xh.numpy(), eps, labels_out=lab_h.numpy()))
    assert np.array_equal(lab_d.cpu().numpy(), lab_h.numpy()), "device and host-buffer runs disagree"

    # profiled run: every kernel group bracketed by CUDA events on its stream
    _, pinfo = egg_sync(Xd, eps, labels_out=lab_d, profile=True)
    grid = grid_leg(Xd, eps, dev, flush) if world == 1 else None
    learned = learned_leg(args, timed, Xd, eps, lab_d, dev) if world == 1 and not args.no_extra else None
    sweep = batched_sweep(dev) if world == 1 and not args.no_extra else None
    mdl = mdl_leg(dev) if world == 1 and not args.no_extra else None

    ms = statistics.mean(dev_times)
    ms_e2e = statistics.mean(e2e_times)
    t_max, t_e2e_max = max_over_ranks(pg, [ms, ms_e2e], dev)
    if rank != 0:
        return None

    iters = info["iterations"]
    upd_ms = pinfo["kernel_ms"]["update"] / max(pinfo["kernel_launches"]["update"], 1)
    peak, peak_kind = measured_peaks()
    # cells per launch differ across iterations; use the mean over the run
    cells = info["n_cells"]
    ub = update_bytes_per_launch(n, d, cells)
    achieved = ub / (upd_ms * 1e-3) / 1e9
    tot_k = sum(pinfo["kernel_ms"].values())
    sample = args.cpu_sample or CPU_SAMPLE
    line = {
        "metric": METRIC,
        "value": t_max / 1000.0,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_max,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "n": n, "d": d, "eps": eps, "iterations": iters,
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "flushed before every timed step (256 MiB write)"},
        "e2e": {"value": t_e2e_max / 1000.0, "unit": "s", "h2d_bytes_per_step": int(n * d * 4),
                "d2h_bytes_per_step": int(n * 4)},
        "gpu_launches": int(info["launches"]) * args.steps,
        "roofline": {"bound": "hbm", "kernel": "k_update", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": UPDATE_DRAM_BYTES_PER_LAUNCH,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, mean of the update "
                                       "launches of iterations 2-4 (-s 193 -c 3), cold cache",
                     "peak_source": peak_kind, "launch_ms": upd_ms,
                     "launches": pinfo["kernel_launches"]["update"],
                     "algorithmic_bytes_per_launch": ub,
                     "share_of_kernel_time": pinfo["kernel_ms"]["update"] / tot_k if tot_k else None},
        "kernel_ms": pinfo["kernel_ms"],
        "stage_ms": info["stage_ms"],
        "clocks": clocks,
        "cpu_baseline": cpu_baseline(X, eps, sample),
    }
    if grid is not None:
        line["roofline_grid"] = grid
        line["roofline_update_fp32"] = update_fp32_leg(args, pinfo["kernel_ms"]["update"])
    if learned is not None:
        line["learned"] = learned
    if sweep is not None:
        line["batched_sweep"] = sweep
    if mdl is not None:
        line["mdl_search"] = mdl
    return line


def ari(a, b):
    """Adjusted Rand index of two labelings (every label value is a group)."""
    a = np.asarray(a, np.int64)
    b = np.asarray(b, np.int64)
    _, ai = np.unique(a, return_inverse=True)
    _, bi = np.unique(b, return_inverse=True)
    pairs = ai * (bi.max() + 1) + bi
    _, nij = np.unique(pairs, return_counts=True)
    comb = lambda x: (x.astype(np.float64) * (x - 1) / 2).sum()  # noqa: E731
    sij = comb(nij)
    sa = comb(np.bincount(ai))
    sb = comb(np.bincount(bi))
    expected = sa * sb / comb(np.array([len(a)]))
    mx = (sa + sb) / 2
    return 1.0 if mx == expected else float((sij - expected) / (mx - expected))


def learned_leg(args, timed, Xd, eps, lab_plain, dev):
    """The learned warm start on the same workload: unverified time, its
    iterations and the agreement of its partition with the plain run's."""
    import torch

    from eggsync import egg_sync, warm

    model = warm.default_model(Xd.shape[1])
    if model is None:
        return {"unavailable": "no trained warm-start model for d = %d" % Xd.shape[1]}
    lab_w = torch.empty_like(lab_plain)
    for _ in range(max(args.warmup, 1)):
        egg_sync(Xd, eps, labels_out=lab_w, warm_start=model)
    times, (_, info) = timed(lambda: egg_sync(Xd, eps, labels_out=lab_w, warm_start=model))
    a, b = lab_plain.cpu().numpy(), lab_w.cpu().numpy()
    _, vinfo = egg_sync(Xd, eps, labels_out=lab_w, warm_start=model, warm_verify=True)
    return {"value": statistics.mean(times) / 1000.0, "unit": "s", "iterations": info["iterations"],
            "warm_ms": info["warm_ms"], "ari_vs_plain": ari(a, b),
            "same_partition_as_plain": bool(vinfo["warm_same"]), "verified_fallback": bool(vinfo["warm_fallback"]),
            "model": "eggsync/models/warm_d3.npz (K=%d, min_count %d)" % (model.k_steps, model.min_count),
            "note": "unverified warm start; with warm_verify the call returns the plain partition when they differ"}


def batched_sweep(dev):
    """C4: 64 datasets x 8 eps (512 runs) in one egg_sync_batch call against
    512 sequential egg_sync calls; device inputs and outputs, wall clock
    around each call after a synchronize."""
    import time

    import torch

    from eggsync import data, egg_sync, egg_sync_batch

    inst = [(torch.from_numpy(c["X"]).to(dev), e) for c in data.c4(0) for e in c["eps"]]
    ob = [torch.empty(len(x), dtype=torch.int32, device=dev) for x, _ in inst]
    os_ = [torch.empty(len(x), dtype=torch.int32, device=dev) for x, _ in inst]
    res, bi = egg_sync_batch(inst, labels_out=ob)  # tunes once (cached)
    tb = []
    for _ in range(3):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        res, bi = egg_sync_batch(inst, labels_out=ob)
        torch.cuda.synchronize(dev)
        tb.append(time.perf_counter() - t0)
    for x, e in inst[:8]:
        egg_sync(x, e)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    sres = [egg_sync(x, e, labels_out=o) for (x, e), o in zip(inst, os_)]
    torch.cuda.synchronize(dev)
    ts = time.perf_counter() - t0
    # device time of the sequential calls (each call's CUDA events from its
    # first to its last operation); the rest of the wall clock is host work:
    # capturing and instantiating each call's loop graph, launches, syncs
    seq_dev = sum(q[1]["total_ms"] for q in sres) / 1000.0
    same = all(torch.equal(a, b) for a, b in zip(ob, os_)) and all(
        r[1]["iterations"] == q[1]["iterations"] for r, q in zip(res, sres))
    return {"workload": "c4: 64 datasets (n 1k-200k, d in {2,3,5}) x 8 eps in [0.01, 0.08], 512 runs",
            "batched_s": min(tb), "sequential_s": ts, "speedup": ts / min(tb), "identical_to_sequential": same,
            "sequential_device_s": seq_dev, "sequential_host_s": ts - seq_dev,
            "loop_iterations": bi["loop_iterations"], "launch_config": {k: bi[k] for k in (
                "update_threads", "blocks_per_sm", "order")}}


def mdl_leg(dev):
    """The MDL eps search (Sync, python/SynCTorch.py:349-372) on 100k x 3D
    (the first 100k points of the c2 shape), k = 5: the brute-force k-NN
    kernel against the FP32 CUDA-core peak, one coding cost, and a search
    capped at 16 candidates; device inputs, CUDA events around each call."""
    import torch

    from eggsync import data, egg_sync, knn_mean, mdl_cost, mdl_search

    X = torch.from_numpy(data.c2(0)["X"][:100_000].copy()).to(dev)
    n, d = X.shape
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, reps):
        fn()
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize(dev)
            ev[0].record()
            out = fn()
            ev[1].record()
            torch.cuda.synchronize(dev)
            ts.append(ev[0].elapsed_time(ev[1]))
        return min(ts), out

    knn_ms, nn = timed(lambda: knn_mean(X, 5), 3)
    lab, _ = egg_sync(X, 0.02)
    cost_ms, (cost, K) = timed(lambda: mdl_cost(X, lab), 3)
    search_ms, (_, info) = timed(lambda: mdl_search(X, 5, max_candidates=16), 1)
    # per pair: d subtractions and d fused multiply-adds (3d FLOP)
    flops = float(n) * n * 3 * d
    fp32_peak = 148 * 128 * 2 * 1.965e9  # nominal FP32 CUDA-core FLOP/s at the max SM clock
    return {"workload": "100k x 3D (c2 shape, first 100k points), k = 5, at most 16 candidates",
            "knn_ms": knn_ms, "knn_pairs_per_s": n * n / (knn_ms * 1e-3),
            "knn_roofline": {"bound": "fp32", "achieved": flops / (knn_ms * 1e-3) / 1e12,
                             "peak": fp32_peak / 1e12, "unit": "TFLOP/s",
                             "frac": flops / (knn_ms * 1e-3) / fp32_peak, "peak_source": "nominal"},
            "nn_k": nn[0], "nn_k1": nn[1], "cost_ms": cost_ms, "cost": cost, "cost_clusters": K,
            "search_ms": search_ms, "candidates": info["candidates"], "best": info["best"],
            "eps_best": info["eps_best"], "n_clusters": info["n_clusters"], "end_reason": info["end_reason"]}


def run_reference(args, rank, world):
    """The reference's own CPU SynC on the box's host cores (rank 0 only):
    every step times one iteration of the same fixed sample as the
    cpu_baseline leg and extrapolates to the whole run."""
    if rank != 0:
        return None
    sys.path.insert(0, str(REPO / "oracle"))
    from eggsync import data
    from oracle import RefSync

    c = data.c5(args.seed, n=args.n)
    X, eps = c["X"], c["eps"]
    sample = args.cpu_sample or CPU_SAMPLE
    R = RefSync()
    vals = []
    dts = []
    for k in range(args.warmup + args.steps):
        per_iter, dt = cpu_iteration_time(R, X, eps, sample)
        if k >= args.warmup:
            vals.append(per_iter * C5_SYNC_ITERATIONS)
            dts.append(dt)
    v = statistics.mean(vals)
    cb = cpu_baseline(X, eps, sample)
    cb["value"] = v
    cb["sample"] = ("reference SynC parallel (OpenMP): per step one iteration of %d sampled points (seed 0) against "
                    "all %d, mean %.2f s over %d steps; extrapolated x n/sample x %d iterations (the CPU SynC's own "
                    "count on this workload)" % (sample, len(X), statistics.mean(dts), args.steps,
                                                 C5_SYNC_ITERATIONS))
    n, d = X.shape
    return {
        "metric": METRIC, "value": v, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": v * 1000.0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
        "config": {"workload": WORKLOAD, "n": n, "d": d, "eps": eps},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def sync_iterations(args):
    """Iterations the reference CPU SynC (SynC.cpp:268-326: lambda stop rule
    on the mean local order parameter, exact eps neighbourhoods) takes on the
    workload, counted with this library's brute-force GPU SynC, which follows
    the same rule (egg_simple_sync_run)."""
    import torch

    from eggsync import data, simple_sync

    dev = torch.device("cuda", 0)
    c = data.c5(args.seed, n=args.n)
    Xd = torch.from_numpy(c["X"]).to(dev)
    t0 = time.perf_counter()
    lab, info = simple_sync(Xd, c["eps"], c["lam"], max_iter=args.sync_max_iter)
    print(json.dumps({"sync_iterations": info["iterations"], "converged": info["converged"],
                      "r_local": info["r_local"], "s": time.perf_counter() - t0, "n": len(c["X"])}))


def main():
    args = parse()
    if args.profile_run:
        profile_run(args)
        return
    if args.profile_grid:
        profile_grid(args)
        return
    if args.stage_split:
        stage_split(args)
        return
    if args.profile_warm:
        profile_warm(args)
        return
    if args.sync_iterations:
        sync_iterations(args)
        return
    rank, local, world, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            line = run_reference(args, rank, world)
        else:
            line = run_ours(args, rank, local, world, pg)
        if line is not None:
            print(json.dumps(line))
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
