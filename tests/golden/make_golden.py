"""Generate the golden fixtures under tests/golden/ from the reference itself.

Two parts, both running the reference's own code built from its sources by
oracle/build.py (oracle/_ref/):

  --cpu   reference CPU SynC (src/algorithms/SynC.cpp), runs anywhere:
          ref_sync_c1.npz   one-iteration update of every point of the c1
                            workload (ComputeNeighborhood + UpdatePoint +
                            ComputeLocationOrder, SynC.cpp:16-56) and the
                            full-run labels / iterations of
                            DynamicalClustering_parallel (SynC.cpp:328-399).
  --gpu   reference EGG-SynC (src/algorithms/EGG_SynC.cu), needs a CUDA
          device; each case is run three times in a child process:
          ref_egg_<case>.npz labels of every run, iteration counts.
  --gpu-simple  reference brute-force GPU SynC (src/algorithms/
          simple_GPU_SynC.cu), needs a CUDA device; each case run twice:
          ref_simple_<case>.npz labels of every run, iteration counts.

Inputs are regenerated from their seeds by eggsync.data / the small cases
below; each fixture stores a checksum of its input so drift is caught.
The reference EGG-SynC is only run on inputs with n <= 32768 (its pair list
is sized with int arithmetic, EGG_SynC.cu:878, 1449-1450) and with at least
one outer grid dimension (with zero it indexes idxs[-1], EGG_SynC.cu:416).

Usage: python tests/golden/make_golden.py --cpu [--gpu] [--out DIR]
"""
from __future__ import annotations

import argparse
import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO / "egg-sync_b200"))
sys.path.insert(0, str(REPO / "oracle"))

from eggsync import data  # noqa: E402


def checksum(X):
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(X, np.float32).tobytes()).digest()[:8], np.uint64)[0]


def small_cases():
    """Adversarial inputs (all n <= 32768 and with od >= 1)."""
    out = {}
    rng = np.random.default_rng(7)
    side = np.float32(np.sqrt((0.05 / 2) ** 2 / 2))
    # points exactly on cell borders, plus the 0 and 1 edges
    k = rng.integers(0, 56, size=(1500, 2)).astype(np.float32)
    X = np.clip(k * side, 0, 1).astype(np.float32)
    X[:20] = 1.0
    X[20:40] = 0.0
    out["borders"] = (X, 0.05)
    # many duplicates around a few sites
    sites = rng.uniform(0.1, 0.9, (6, 2)).astype(np.float32)
    X = sites[rng.integers(0, 6, 3000)] + (rng.random((3000, 2)) < 0.1) * rng.normal(0, 0.01, (3000, 2))
    out["duplicates"] = (data.min_max_normalize(X), 0.05)
    # d = 1
    X = data.blobs(rng, 2000, 1, rng.uniform(0.1, 0.9, (5, 1)), [0.02] * 5, np.ones(5), 0.05)
    out["d1"] = (X, 0.05)
    # small n (od = 1)
    X = data.blobs(rng, 300, 2, rng.uniform(0.1, 0.9, (4, 2)), [0.03] * 4, np.ones(4), 0.1)
    out["n300"] = (X, 0.05)
    # uniform noise only
    out["noise"] = (data.min_max_normalize(rng.random((4000, 2))), 0.02)
    # d = 5
    X = data.blobs(rng, 6000, 5, rng.uniform(0.1, 0.9, (8, 5)), [0.03] * 8, np.ones(8), 0.05)
    out["d5"] = (X, 0.08)
    return out


def gpu_cases():
    cases = {}
    for s in (0, 1, 2):
        c = data.c1(s)
        cases["c1_s%d" % s] = (c["X"], c["eps"])
    c = data.c3a(0)
    cases["c3a_s0"] = (c["X"], c["eps"])
    cases.update(small_cases())
    return cases


def make_cpu(out: Path):
    from oracle import RefSync

    R = RefSync()
    c = data.c1(0)
    X, eps = c["X"], c["eps"]
    idx = np.arange(len(X), dtype=np.int32)
    step, counts, r = R.step_sample(X, eps, idx)
    labels, iters = R.run(X, eps, c["lam"])
    np.savez_compressed(out / "ref_sync_c1.npz", x_checksum=checksum(X), eps=np.float32(eps), step=step,
                        counts=counts, r_local=r, labels=labels, iterations=np.int32(iters),
                        threads=np.int32(R.threads()))
    print("ref_sync_c1.npz: iterations", iters)


def make_gpu(out: Path, runs=3):
    from oracle import run_ref_egg

    for name, (X, eps) in gpu_cases().items():
        labs, its = [], []
        for _ in range(runs):
            lab, it, _st = run_ref_egg(X, eps, timeout=900)
            labs.append(lab)
            its.append(it)
        np.savez_compressed(out / ("ref_egg_%s.npz" % name), x_checksum=checksum(X), eps=np.float32(eps),
                            labels=np.stack(labs), iterations=np.array(its, np.int32))
        print("ref_egg_%s.npz: n=%d iterations %s" % (name, len(X), its))


def simple_cases():
    """Inputs of the brute-force drop-in's fixtures (small: O(n^2) per iteration)."""
    out = {}
    for seed in (0, 1):
        out["c1_%d" % seed] = (np.ascontiguousarray(data.c1(seed)["X"][:3000]), 0.05)
    rng = np.random.default_rng(3)
    out["blobs3d"] = (data.blobs(rng, 2000, 3, rng.uniform(0.2, 0.8, (4, 3)), [0.03] * 4, np.ones(4), 0.05), 0.08)
    return out


def make_gpu_simple(out: Path, runs=2):
    """Labels and iteration counts of the reference's own GPU_DynamicalClustering."""
    from oracle import run_ref_simple

    for name, (X, eps) in simple_cases().items():
        labs, its = [], []
        for _ in range(runs):
            lab, it = run_ref_simple(X, eps, timeout=900)
            labs.append(lab)
            its.append(it)
        np.savez_compressed(out / ("ref_simple_%s.npz" % name), x_checksum=checksum(X), eps=np.float32(eps),
                            labels=np.stack(labs), iterations=np.array(its, np.int32))
        print("ref_simple_%s.npz: n=%d iterations %s" % (name, len(X), its))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--cpu", action="store_true")
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--gpu-simple", action="store_true")
    ap.add_argument("--out", default=str(HERE))
    a = ap.parse_args()
    o = Path(a.out)
    o.mkdir(parents=True, exist_ok=True)
    if a.cpu:
        make_cpu(o)
    if a.gpu:
        make_gpu(o)
    if a.gpu_simple:
        make_gpu_simple(o)
