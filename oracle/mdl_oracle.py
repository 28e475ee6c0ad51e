"""CPU restatement of the MDL eps search (TEST INFRASTRUCTURE ONLY).

Only ``tests/`` import this module; it is the checker of the CUDA path in
``egg-sync_b200/csrc/egg_mdl.cu``, never part of it.  Pinned against the
reference's own functions run on small inputs (``tests/golden/ref_mdl.npz``,
made by ``tests/golden/make_mdl_golden.py``).

* ``nn_mean(X, k)``: python/SynCTorch.py:112-137 (NN): mean over the points
  of the distance to the k-th nearest other point.
* ``bandwidths(X)``: SynCTorch.py:284-286: h_l = 0.9 n^(-1/(d+4))
  min(var_l, IQR_l / 1.34), var unbiased (the reference's ``sigma`` is
  ``torch.var``), IQR = 75th - 25th percentile, linear interpolation
  (``scipy.stats.iqr``).
* ``mdl_cost(X, labels)``: SynCTorch.py:265-314 (L_Clust_Outl) for the
  clustering whose clusters are the points sharing a label >= 0 and whose
  outliers carry label -1.
* ``search(X, k, cluster, max_candidates)``: SynCTorch.py:349-372 (Sync)
  with a given clustering function eps -> labels.
All in float64 from the float32 inputs.
"""
from __future__ import annotations

import numpy as np


def nn_mean(X, k):
    X = np.asarray(X, np.float64)
    n = len(X)
    sq = ((X[:, None, :] - X[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(sq, np.inf)
    kth = np.partition(sq, k - 1, axis=1)[:, k - 1]
    return float(np.sqrt(kth).mean())


def bandwidths(X):
    X = np.asarray(X, np.float64)
    n, d = X.shape
    var = X.var(axis=0, ddof=1)
    q75, q25 = np.percentile(X, [75, 25], axis=0)
    return 0.9 * n ** (-1.0 / (d + 4)) * np.minimum(var, (q75 - q25) / 1.34)


def clusters_of(labels):
    labels = np.asarray(labels)
    return [np.nonzero(labels == c)[0] for c in np.unique(labels[labels >= 0])]


def mdl_cost(X, labels):
    X = np.asarray(X, np.float64)
    n, d = X.shape
    h = bandwidths(X)
    cl = clusters_of(labels)
    outliers = n - sum(len(c) for c in cl)
    lm = sum(len(c) * np.log2(n / len(c)) + d / 2 * np.log2(len(c)) for c in cl) + outliers * np.log2(n)
    norm = (2 * np.pi) ** (-d / 2) / np.prod(h)
    ld = 0.0
    for c in cl:
        P = X[c] / h
        sq = ((P[:, None, :] - P[None, :, :]) ** 2).sum(-1)
        f = norm * np.exp(-0.5 * sq).sum(1) / len(c)
        ld += np.log2(f / f.sum()).sum()
    ld += outliers * (2 * np.pi) ** -0.5 * np.prod(h)
    return float(lm - ld)


def eps_schedule(nn_k, nn_k1, count):
    """eps = NN(k); delta = NN(k+1) - eps; eps += delta, in float32."""
    e = np.float32(nn_k)
    step = np.float32(nn_k1) - e
    out = []
    for _ in range(count):
        out.append(e)
        e = np.float32(e + step)
    return np.array(out, np.float32), step


def search(X, k, cluster, max_candidates=256):
    """(best index, costs, eps values, cluster counts) of the search;
    cluster(eps) returns labels."""
    eps, _ = eps_schedule(nn_mean(X, k), nn_mean(X, k + 1), max_candidates)
    costs, ks = [], []
    for e in eps:
        lab = cluster(float(e))
        costs.append(mdl_cost(X, lab))
        ks.append(len(clusters_of(lab)))
        if ks[-1] == 1:
            break
    return int(np.argmin(costs)), np.array(costs), eps[:len(costs)], np.array(ks)
