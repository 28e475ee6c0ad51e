"""Golden fixtures of the reference EGG-SynC at the large workloads.

For each of the 250k x 3 (eps 0.03), 500k x 3 (eps 0.02) and 1M x 3
(eps 0.015) workloads (seed 0, eggsync.data):

1. The trajectory is followed with this library's one-iteration entry
   point (egg_sync_step); in every iteration whose update leaves the
   convergence flag set, which is when the reference runs its extra check,
   the number of pairs the reference's extra check lists is counted on the
   CPU (Oracle.ref_annulus_pairs, EGG_SynC.cu:767-878).
2. The reference sizes that pair list with int arithmetic (EGG_SynC.cu:878,
   1010, 1449-1450).  Only when every count stays below
   oracle.ref_egg_pair_limit(n) is the reference itself run (child process,
   wall-clock timeout), and its labels, iteration count and wall time are
   stored in ref_egg_<name>.npz.  Otherwise the counts are stored with
   ref_ran = 0 and the reason.

Needs a CUDA device and oracle/_ref/libref_egg.so (oracle/build.py).

    python tests/golden/make_golden_large.py [--only c3b_s0,c2_s0] [--no-ref] [--timeout S]
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO / "egg-sync_b200"))
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(HERE))

from eggsync import data, egg_step, egg_sync  # noqa: E402
from make_golden import checksum  # noqa: E402


def large_cases():
    out = {}
    for name, fn in (("c3b_s0", data.c3b), ("c2_s0", data.c2), ("c5_s0", data.c5)):
        c = fn(0)
        out[name] = (c["X"], c["eps"])
    return out


def annulus_counts(O, X, eps, max_iter=1000):
    """[(iteration, total pairs, largest per point)] over the iterations
    whose update flag is set, and the iteration count of the step chain."""
    x = X
    rows = []
    for it in range(max_iter):
        xn, _cnt, flags = egg_step(x, eps)
        if flags[0]:
            total, worst = O.ref_annulus_pairs(x, eps)
            rows.append((it, total, worst))
        if flags[1]:
            return rows, it + 1
        x = xn
    return rows, max_iter


def main():
    from oracle import Oracle, ari, ref_egg_pair_limit, run_ref_egg

    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="")
    ap.add_argument("--no-ref", action="store_true")
    ap.add_argument("--timeout", type=float, default=1200.0)
    ap.add_argument("--ref-runs", type=int, default=1, help="runs of the reference per workload")
    ap.add_argument("--save-ours", default="", help="folder for this library's labels (inspection)")
    ap.add_argument("--out", default=str(HERE))
    a = ap.parse_args()
    O = Oracle()
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    only = set(a.only.split(",")) if a.only else None
    for name, (X, eps) in large_cases().items():
        if only and name not in only:
            continue
        n = len(X)
        t0 = time.time()
        rows, chain_iters = annulus_counts(O, X, eps)
        t_count = time.time() - t0
        limit = ref_egg_pair_limit(n)
        worst_total = max([r[1] for r in rows], default=0)
        safe = worst_total < limit
        lab, info = egg_sync(X, eps)
        rec = {"name": name, "n": n, "eps": eps, "chain_iterations": chain_iters, "extra_check_iterations": len(rows),
               "max_pairs": worst_total, "pair_limit": limit, "safe": safe, "count_s": round(t_count, 1),
               "iterations": info["iterations"], "ms": info["total_ms"]}
        fields = dict(x_checksum=checksum(X), eps=np.float32(eps),
                      pair_rows=np.array(rows, np.int64).reshape(-1, 3), pair_limit=np.int64(limit),
                      iterations_here=np.int32(info["iterations"]))
        if a.save_ours:
            Path(a.save_ours).mkdir(parents=True, exist_ok=True)
            np.save(Path(a.save_ours) / ("labels_%s.npy" % name), lab)
        if safe and not a.no_ref:
            labs, its, walls = [], [], []
            for _ in range(a.ref_runs):
                ref_info = {}
                rlab, rit, _st = run_ref_egg(X, eps, timeout=a.timeout, max_pairs=worst_total, info_out=ref_info)
                labs.append(rlab.astype(np.int32))
                its.append(rit)
                walls.append(ref_info.get("wall_s", -1.0))
            rec.update(ref_iterations=its, ref_wall_s=walls, ari=[ari(lab, r) for r in labs],
                       ref_ari_between_runs=[ari(labs[0], r) for r in labs[1:]],
                       same_iterations=all(i == info["iterations"] for i in its))
            fields.update(ref_ran=np.int32(1), labels=np.stack(labs), iterations=np.array(its, np.int32),
                          ref_wall_s=np.array(walls, np.float64))
        else:
            fields.update(ref_ran=np.int32(0),
                          reason=np.array("pair count %d not below the reference's limit %d" % (worst_total, limit)
                                          if not safe else "reference not run (--no-ref)"))
        np.savez_compressed(out / ("ref_egg_%s.npz" % name), **fields)
        print("LARGE_GOLDEN " + json.dumps(rec), flush=True)


if __name__ == "__main__":
    main()
