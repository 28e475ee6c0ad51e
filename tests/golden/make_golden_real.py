"""Golden fixtures of the reference EGG-SynC on the reference's own real
data sets (python/data.py:44-97), min-max normalised, eps 0.05
(run_experiment.py:547-551).

The data files are read from a copy of the reference's data/ folder (first
argument, or EGG_REAL_DATA, or _data/real in the repository); only the
reference's labels (canonical numbering: clusters numbered by first
occurrence, -1 kept) and iteration counts are stored, in
ref_egg_real_<name>.npz.  Above 32,768 points the reference's extra-check
pair count is checked against its int limits first, as in
make_golden_large.py.  Needs a CUDA device and oracle/_ref/libref_egg.so.

    python tests/golden/make_golden_real.py [DATA_DIR] [--out DIR]
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO / "egg-sync_b200"))
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(HERE))

from eggsync import data, egg_sync  # noqa: E402
from make_golden import checksum  # noqa: E402
from make_golden_large import annulus_counts  # noqa: E402


def canonical(lab):
    lab = np.asarray(lab, np.int64)
    u, first = np.unique(lab[lab >= 0], return_index=True)
    order = np.argsort(first)
    lut = np.full(int(lab.max()) + 2 if lab.size else 1, -1, np.int64)
    lut[u[order]] = np.arange(len(u))
    return np.where(lab >= 0, lut[np.maximum(lab, 0)], -1).astype(np.int32)


def main():
    from oracle import REF_EGG_MAX_N, Oracle, ari, ref_egg_pair_limit, run_ref_egg

    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    out = Path(sys.argv[sys.argv.index("--out") + 1]) if "--out" in sys.argv else HERE
    if args and args[0] == str(out):
        args = args[1:]
    src = Path(args[0] if args else os.environ.get("EGG_REAL_DATA", str(REPO / "_data" / "real")))
    out.mkdir(parents=True, exist_ok=True)
    O = Oracle()
    eps = data.REAL_EPS
    for name in sorted(data.REAL):
        X = data.load_real(name, src)
        n = len(X)
        max_pairs = None
        if n > REF_EGG_MAX_N:
            rows, _ = annulus_counts(O, X, eps)
            max_pairs = max([r[1] for r in rows], default=0)
            if max_pairs >= ref_egg_pair_limit(n):
                print("REAL_GOLDEN " + json.dumps({"name": name, "skipped": "pair count %d" % max_pairs}))
                continue
        labs, its, walls = [], [], []
        for _ in range(2):
            info = {}
            lab, it, _ = run_ref_egg(X, eps, timeout=1200, max_pairs=max_pairs, info_out=info)
            labs.append(canonical(lab))
            its.append(it)
            walls.append(info.get("wall_s", -1.0))
        same = all(np.array_equal(labs[0], x) for x in labs[1:])
        ours, oi = egg_sync(X, eps)
        np.savez_compressed(out / ("ref_egg_real_%s.npz" % name), x_checksum=checksum(X), eps=np.float32(eps),
                            labels=labs[0][None, :], iterations=np.array(its, np.int32),
                            ref_wall_s=np.array(walls), ref_runs_same_partition=np.int32(same))
        print("REAL_GOLDEN " + json.dumps({"name": name, "n": n, "d": X.shape[1], "ref_iterations": its,
                                           "ref_wall_s": walls, "runs_same": same, "ours_iterations": oi["iterations"],
                                           "ours_ms": oi["total_ms"], "ari": ari(ours, labs[0])}), flush=True)


if __name__ == "__main__":
    main()
