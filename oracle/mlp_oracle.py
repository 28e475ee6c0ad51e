"""CPU restatement of the learned warm start (TEST INFRASTRUCTURE ONLY).

The warm start has no counterpart in the reference: this module restates the
library's own specification of it in numpy so that the tests can check the
CUDA kernels (``egg-sync_b200/csrc/egg_mlp.cu``) against it.  Only
``tests/`` import it.  It is pinned by a finite-difference check of
``grad`` (``tests/test_warm_oracle.py``); parity of the final labels with
the plain loop is checked directly on the GPU.

* ``features``: the coarse grid of side eps with fixed-point (2^24) sums of
  the in-cell offsets, the per-point row layout (offset, then per neighbour
  cell in {-1,0,1}^d with the first dimension fastest: log1p(count)/8,
  centroid - point, spread), zero padding to a multiple of 16.
* ``forward``: the 3-layer MLP (ReLU), either in float64 or with the
  kernel's BF16 rounding of the operands and of the hidden activations.
* ``grad``: float64 mean-squared-error gradient of one batch.
"""
from __future__ import annotations

import numpy as np

FIX = np.float32(16777216.0)
NAMES = ("w1", "b1", "w2", "b2", "w3", "b3")


def feature_dim(d):
    return d + 3 ** d * (1 + 2 * d)


def feature_width(d):
    return (feature_dim(d) + 15) // 16 * 16


def _coarse(X, eps):
    f = np.float32(eps)
    width = max(1, int(np.ceil(1.0 / float(f))))  # from the float32 eps, as the kernels
    q = (X / f).astype(np.float32)
    c = np.clip(q.astype(np.int64), 0, width - 1)
    u = (q - c.astype(np.float32)).astype(np.float32)
    return c, u, width


def features(X, eps):
    X = np.asarray(X, np.float32)
    n, d = X.shape
    c, u, width = _coarse(X, eps)
    mul = width ** np.arange(d)
    cell = (c * mul).sum(1)
    U = np.rint((u * FIX).astype(np.float32)).astype(np.int64)
    Q = np.rint((u * u * FIX).astype(np.float32)).astype(np.int64)
    ncell = width ** d
    cnt = np.bincount(cell, minlength=ncell)
    su = np.zeros((ncell, d), np.int64)
    sq = np.zeros((ncell, d), np.int64)
    for l in range(d):
        np.add.at(su[:, l], cell, U[:, l])
        np.add.at(sq[:, l], cell, Q[:, l])
    out = np.zeros((n, feature_width(d)), np.float32)
    out[:, :d] = u
    k = d
    for s in range(3 ** d):
        o = np.array([(s // 3 ** l) % 3 - 1 for l in range(d)])
        v = c + o
        inb = ((v >= 0) & (v < width)).all(1)
        vc = (np.clip(v, 0, width - 1) * mul).sum(1)
        m = np.where(inb, cnt[vc], 0)
        has = m > 0
        out[has, k] = (np.log1p(m[has].astype(np.float32)) * np.float32(0.125)).astype(np.float32)
        mm = np.maximum(m, 1).astype(np.float64)[:, None]
        mean = su[vc] / (mm * float(FIX))
        e2 = sq[vc] / (mm * float(FIX))
        var = np.maximum(0.0, e2 - mean * mean)
        rel = (mean + o[None, :] - u.astype(np.float64)).astype(np.float32)
        out[has, k + 1:k + 1 + d] = rel[has]
        out[has, k + 1 + d:k + 1 + 2 * d] = np.sqrt(var[has]).astype(np.float32)
        k += 1 + 2 * d
    return out


def bf16(a):
    """Round float32 to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def forward(w, feats, d, emulate_bf16=False):
    F = feature_dim(d)
    x = np.asarray(feats)[:, :F]
    if emulate_bf16:
        h1 = np.maximum(bf16(x.astype(np.float32)).astype(np.float64) @ bf16(w["w1"]).astype(np.float64) + w["b1"], 0)
        h1 = bf16(h1.astype(np.float32)).astype(np.float64)
        h2 = np.maximum(h1 @ bf16(w["w2"]).astype(np.float64) + w["b2"], 0)
        h2 = bf16(h2.astype(np.float32)).astype(np.float64)
        return h2 @ bf16(w["w3"]).astype(np.float64) + w["b3"]
    x = x.astype(np.float64)
    h1 = np.maximum(x @ w["w1"] + w["b1"], 0)
    h2 = np.maximum(h1 @ w["w2"] + w["b2"], 0)
    return h2 @ w["w3"] + w["b3"]


def grad(w, feats, targets, d):
    """(mean squared error, gradients) in float64."""
    F = feature_dim(d)
    x = np.asarray(feats, np.float64)[:, :F]
    t = np.asarray(targets, np.float64)
    W = {k: np.asarray(v, np.float64) for k, v in w.items()}
    a1 = x @ W["w1"] + W["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W["w2"] + W["b2"]
    h2 = np.maximum(a2, 0)
    y = h2 @ W["w3"] + W["b3"]
    e = y - t
    loss = (e ** 2).mean()
    dy = 2 * e / e.size
    g = {"w3": h2.T @ dy, "b3": dy.sum(0)}
    dh2 = dy @ W["w3"].T * (a2 > 0)
    g["w2"], g["b2"] = h1.T @ dh2, dh2.sum(0)
    dh1 = dh2 @ W["w2"].T * (a1 > 0)
    g["w1"], g["b1"] = x.T @ dh1, dh1.sum(0)
    return loss, g


def mse(w, feats, targets, d):
    y = forward(w, feats, d)
    return ((y - np.asarray(targets, np.float64)) ** 2).mean()
