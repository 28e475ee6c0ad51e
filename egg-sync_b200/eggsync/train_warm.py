"""Train the warm-start network on trajectories of the plain loop.

    python -m eggsync.train_warm [--instances 200] [--sample 25000] [--k 8]
                                 [--epochs 30] [--out PATH]

Training instances are data.train_instance(seed) for seeds 1,000,000 + i
(100k points in 3-D, 8-40 clusters, 10% noise, eps 0.02); validation uses
seeds 1,500,000 + i.  Targets are the displacement after k iterations of the
plain loop, in eps units.  Every step runs on the GPU through the C ABI
(features, trajectories, FP32 training kernels, BF16 inference for the
validation error).  Prints one JSON line and writes the model (.npz).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import warm


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, default=200)
    ap.add_argument("--val-instances", type=int, default=4)
    ap.add_argument("--sample", type=int, default=25000)
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=2048)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--min-count", type=int, default=300,
                    help="displace only points with this many points in their 3^d coarse cells")
    ap.add_argument("--out", default=str(warm.MODEL_DIR / "warm_d3.npz"))
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    f, t = warm.make_training_set(range(1_000_000, 1_000_000 + a.instances), a.k, a.sample, a.seed)
    fv, tv = warm.make_training_set(range(1_500_000, 1_500_000 + a.val_instances), a.k, a.sample, a.seed + 1)
    t1 = time.perf_counter()
    model = warm.Model(3, k_steps=a.k, seed=a.seed, min_count=a.min_count)
    losses = warm.train(model, f, t, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed)
    t2 = time.perf_counter()
    pv = warm.forward(model, fv)
    val = float(((pv - tv) ** 2).mean())
    zero = float((tv ** 2).mean())
    model.save(a.out)
    print(json.dumps({"samples": len(f), "k": a.k, "epochs": a.epochs, "train_loss_first": losses[0],
                      "train_loss_last": losses[-1], "val_mse": val, "val_mse_zero_prediction": zero,
                      "data_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 2), "out": a.out}))


if __name__ == "__main__":
    main()
