"""Learned warm start for the synchronisation loop (no counterpart in the
reference).

A small MLP (d_in -> 128 -> 128 -> d, ReLU) reads each point's features
(``features``: its offset in a coarse cell of side eps and summaries of the
3^d coarse cells around it) and predicts its displacement over the next K
iterations of the plain loop, in units of eps.  ``egg_sync(..., warm_start=
model)`` displaces the input by that prediction and runs the plain loop from
there to convergence; with ``warm_verify=True`` it also runs the plain loop
from the input and returns the plain result when the partitions differ.

Everything here calls the CUDA kernels of libeggsync.so through the C ABI:
features, BF16 tensor-core inference, FP32 training kernels (Adam).
``make_training_set`` generates (features, target displacement) pairs from
trajectories of the plain loop on training instances (seeds >= 1,000,000,
disjoint from the evaluation seeds).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import EggMlp, EggMlpTrainOpts, check

HIDDEN = 128
MODEL_DIR = Path(__file__).resolve().parent / "models"
NAMES = ("w1", "b1", "w2", "b2", "w3", "b3")


def feature_dim(d: int) -> int:
    """Unpadded feature count d + 3^d (1 + 2d)."""
    return d + 3 ** d * (1 + 2 * d)


def feature_width(d: int) -> int:
    """Row width of ``features``' output (feature_dim rounded up to 16)."""
    return _lib.load().egg_mlp_feature_dim(d)


class Model:
    """Weights of the warm-start network (float32, row-major [in][out])."""

    def __init__(self, d: int, k_steps: int = 8, seed: int = 0, weights=None, min_count: int = 0):
        self.d = int(d)
        self.k_steps = int(k_steps)
        self.min_count = int(min_count)
        F = feature_dim(self.d)
        if weights is None:
            rng = np.random.default_rng(seed)

            def he(i, o):
                return (rng.standard_normal((i, o)) * np.sqrt(2.0 / i)).astype(np.float32)

            weights = {"w1": he(F, HIDDEN), "b1": np.zeros(HIDDEN, np.float32),
                       "w2": he(HIDDEN, HIDDEN), "b2": np.zeros(HIDDEN, np.float32),
                       "w3": (he(HIDDEN, self.d) * 0.1).astype(np.float32), "b3": np.zeros(self.d, np.float32)}
        self.w = {k: np.ascontiguousarray(weights[k], np.float32) for k in NAMES}
        assert self.w["w1"].shape == (F, HIDDEN) and self.w["w3"].shape == (HIDDEN, self.d)

    def struct(self) -> EggMlp:
        m = EggMlp()
        m.d, m.d_in, m.hidden, m.k_steps = self.d, feature_dim(self.d), HIDDEN, self.k_steps
        m.min_count = self.min_count
        for k in NAMES:
            setattr(m, k, self.w[k].ctypes.data)
        return m

    def save(self, path):
        np.savez(path, d=self.d, k_steps=self.k_steps, min_count=self.min_count, **self.w)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        mc = int(z["min_count"]) if "min_count" in z else 0
        return cls(int(z["d"]), int(z["k_steps"]), weights={k: z[k] for k in NAMES}, min_count=mc)

    def copy(self):
        return Model(self.d, self.k_steps, weights={k: v.copy() for k, v in self.w.items()},
                     min_count=self.min_count)


def default_model(d: int = 3):
    """The committed network for dimension d (trained by train_warm.py), or None."""
    p = MODEL_DIR / ("warm_d%d.npz" % d)
    return Model.load(p) if p.exists() else None


def features(X: np.ndarray, eps: float) -> np.ndarray:
    X = np.ascontiguousarray(X, np.float32)
    n, d = X.shape
    out = np.empty((n, feature_width(d)), np.float32)
    check(_lib.load().egg_mlp_features(C.c_void_p(X.ctypes.data), n, d, float(eps), C.c_void_p(out.ctypes.data)))
    return out


def forward(model: Model, feats: np.ndarray) -> np.ndarray:
    """BF16 tensor-core inference: (n, d) displacements in eps units."""
    feats = np.ascontiguousarray(feats, np.float32)
    out = np.empty((len(feats), model.d), np.float32)
    m = model.struct()
    check(_lib.load().egg_mlp_forward(C.byref(m), C.c_void_p(feats.ctypes.data), len(feats),
                                      C.c_void_p(out.ctypes.data)))
    return out


def grad(model: Model, feats: np.ndarray, targets: np.ndarray):
    """(mean squared error, {name: gradient}) of one batch, FP32 kernels."""
    feats = np.ascontiguousarray(feats, np.float32)
    targets = np.ascontiguousarray(targets, np.float32)
    g = Model(model.d, model.k_steps, weights={k: np.zeros_like(v) for k, v in model.w.items()})
    m, gm = model.struct(), g.struct()
    loss = C.c_double(0)
    check(_lib.load().egg_mlp_grad(C.byref(m), C.c_void_p(feats.ctypes.data), C.c_void_p(targets.ctypes.data),
                                   len(feats), C.byref(gm), C.byref(loss)))
    return loss.value, g.w


def train(model: Model, feats: np.ndarray, targets: np.ndarray, epochs: int = 20, batch: int = 1024,
          lr: float = 1e-3, seed: int = 0):
    """Train ``model`` in place; returns the per-epoch mean squared error."""
    feats = np.ascontiguousarray(feats, np.float32)
    targets = np.ascontiguousarray(targets, np.float32)
    o = EggMlpTrainOpts()
    o.epochs, o.batch, o.lr, o.seed = int(epochs), int(batch), float(lr), int(seed)
    losses = (C.c_double * epochs)()
    m = model.struct()
    check(_lib.load().egg_mlp_train(C.byref(m), C.c_void_p(feats.ctypes.data), C.c_void_p(targets.ctypes.data),
                                    len(feats), C.byref(o), losses))
    return [float(v) for v in losses]


def trajectory_pair(X: np.ndarray, eps: float, k_steps: int):
    """(features of X, displacement after k_steps plain iterations in eps units)."""
    from .algorithms import egg_sync

    P = np.empty_like(X)
    egg_sync(X, eps, max_iter=k_steps, positions_out=P)
    return features(X, eps), ((P - X) / np.float32(eps)).astype(np.float32)


def make_training_set(seeds, k_steps: int = 8, sample: int = 0, rng_seed: int = 0):
    """Stack trajectory pairs of data.train_instance(seed) for every seed;
    ``sample`` > 0 keeps that many random rows per instance."""
    from . import data

    rng = np.random.default_rng(rng_seed)
    fs, ts = [], []
    for s in seeds:
        inst = data.train_instance(s)
        f, t = trajectory_pair(inst["X"], inst["eps"], k_steps)
        if sample and sample < len(f):
            idx = rng.choice(len(f), sample, replace=False)
            f, t = f[idx], t[idx]
        fs.append(f)
        ts.append(t)
    return np.concatenate(fs), np.concatenate(ts)


__all__ = ["Model", "default_model", "features", "forward", "grad", "train", "feature_dim", "feature_width",
           "trajectory_pair", "make_training_set", "HIDDEN"]
