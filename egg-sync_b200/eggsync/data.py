"""Seeded synthetic workloads for EGG-SynC (the shapes of the benchmark configs).

The reference draws its synthetic data with sklearn ``make_blobs`` in
[-100, 100] boxes from an unseeded RNG (python/generator.py:174-223,
python/data.py:5-41) and min-max normalises each dimension
(python/data.py:100-103).  These generators keep that last step and the
float32 row-major layout, and draw everything else from
``numpy.random.Generator(PCG64(seed))`` with the shapes below:

* ``c1``  10,000 x 2: 10 isotropic Gaussians, centres U[0.1,0.9]^2, std 0.02,
  equal sizes, 5% uniform noise; eps 0.05.
* ``c2``  500,000 x 3: 20 anisotropic Gaussians, centres U[0.1,0.9]^3, per-axis
  std U[0.005,0.03], sizes Dirichlet(1) over the 90% clustered share, 10%
  noise; eps 0.02.
* ``c3a`` 20,000 x 16: 26 Gaussians, centres U[0.2,0.8]^16, std 0.04, sizes
  uniform +-30% around the mean, no noise; eps 0.15.
* ``c3b`` 250,000 x 3: 2 Gaussians of 20%/80% weight, std 0.05/0.15, centres
  U[0.1,0.9]^3, 5% noise; eps 0.03.
* ``c4``  64 instances, n log-uniform in [1,000, 200,000], d in {2,3,5},
  5-30 Gaussians with std U[0.01,0.04], 5% noise, each at 8 eps log-spaced in
  [0.01, 0.08].
* ``c5``  1,000,000 x 3: 50 Gaussians, centres U[0.1,0.9]^3, per-cluster std
  U[0.005,0.03], equal sizes, 10% noise; eps 0.015.
* ``train`` 100,000 x 3: 8-40 Gaussians, std U[0.005,0.03], 10% noise;
  eps 0.02 (seeds >= 1,000,000, disjoint from evaluation seeds).

Real data sets: the reference's experiments cluster ten UCI-style files from
its ``data/`` directory, min-max normalised, at eps 0.05
(run_experiment.py:12, 53-62, 547-551; loaders python/data.py:44-97; the
Roads file 3D_spatial_network.txt is not shipped with it).  Their points are
not part of this package: ``load_real`` reads those files from a directory
the caller names, with the reference's columns and delimiters, and
``stand_in`` draws seeded points of the same shape (8 Gaussians with std
U[0.02, 0.08], 5% noise), which the tests run through the GPU path.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

LAMBDA = 1 - 1e-3


def min_max_normalize(X):
    """python/data.py:100-103, per dimension, returned as float32."""
    X = np.asarray(X, dtype=np.float64)
    lo = X.min(axis=0)
    hi = X.max(axis=0)
    span = np.where(hi > lo, hi - lo, 1.0)
    return ((X - lo) / span).astype(np.float32)


def _split(total, weights):
    w = np.asarray(weights, np.float64)
    w = w / w.sum()
    sizes = np.floor(w * total).astype(np.int64)
    rem = total - sizes.sum()
    order = np.argsort(-(w * total - sizes), kind="stable")
    sizes[order[:rem]] += 1
    return sizes


def blobs(rng, n, d, centres, stds, weights, noise):
    """Gaussian clusters plus a uniform-noise share, shuffled and normalised."""
    n_noise = int(round(noise * n))
    sizes = _split(n - n_noise, weights)
    parts = []
    for k, m in enumerate(sizes):
        s = np.broadcast_to(np.asarray(stds[k], np.float64), (d,))
        parts.append(centres[k] + rng.standard_normal((int(m), d)) * s)
    if n_noise:
        parts.append(rng.random((n_noise, d)))
    X = np.concatenate(parts, 0)
    X = X[rng.permutation(n)]
    return min_max_normalize(X)


def c1(seed=0):
    rng = np.random.default_rng(seed)
    k, d = 10, 2
    X = blobs(rng, 10_000, d, rng.uniform(0.1, 0.9, (k, d)), [0.02] * k, np.ones(k), 0.05)
    return {"name": "c1", "X": X, "eps": 0.05, "lam": LAMBDA}


def c2(seed=0):
    rng = np.random.default_rng(seed)
    k, d = 20, 3
    centres = rng.uniform(0.1, 0.9, (k, d))
    stds = rng.uniform(0.005, 0.03, (k, d))
    w = rng.dirichlet(np.ones(k))
    X = blobs(rng, 500_000, d, centres, stds, w, 0.10)
    return {"name": "c2", "X": X, "eps": 0.02, "lam": LAMBDA}


def c3a(seed=0):
    rng = np.random.default_rng(seed)
    k, d = 26, 16
    centres = rng.uniform(0.2, 0.8, (k, d))
    w = rng.uniform(0.7, 1.3, k)
    X = blobs(rng, 20_000, d, centres, [0.04] * k, w, 0.0)
    return {"name": "c3a", "X": X, "eps": 0.15, "lam": LAMBDA}


def c3b(seed=0):
    rng = np.random.default_rng(seed)
    d = 3
    centres = rng.uniform(0.1, 0.9, (2, d))
    X = blobs(rng, 250_000, d, centres, [0.05, 0.15], [0.2, 0.8], 0.05)
    return {"name": "c3b", "X": X, "eps": 0.03, "lam": LAMBDA}


def c5(seed=0, n=1_000_000):
    rng = np.random.default_rng(seed)
    k, d = 50, 3
    centres = rng.uniform(0.1, 0.9, (k, d))
    stds = rng.uniform(0.005, 0.03, k)
    X = blobs(rng, n, d, centres, stds, np.ones(k), 0.10)
    return {"name": "c5", "X": X, "eps": 0.015, "lam": LAMBDA}


def train_instance(seed):
    """One training trajectory instance (use seeds >= 1,000,000)."""
    rng = np.random.default_rng(seed)
    d = 3
    k = int(rng.integers(8, 41))
    centres = rng.uniform(0.1, 0.9, (k, d))
    stds = rng.uniform(0.005, 0.03, k)
    X = blobs(rng, 100_000, d, centres, stds, np.ones(k), 0.10)
    return {"name": "train", "X": X, "eps": 0.02, "lam": LAMBDA}


C4_EPS = np.logspace(np.log10(0.01), np.log10(0.08), 8).astype(np.float32)


def c4(seed=0, instances=64):
    """List of (X, [eps...]) for the batched eps sweep."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(instances):
        n = int(round(np.exp(rng.uniform(np.log(1_000), np.log(200_000)))))
        d = int(rng.choice([2, 3, 5]))
        k = int(rng.integers(5, 31))
        centres = rng.uniform(0.1, 0.9, (k, d))
        stds = rng.uniform(0.01, 0.04, k)
        X = blobs(rng, n, d, centres, stds, np.ones(k), 0.05)
        out.append({"X": X, "eps": [float(e) for e in C4_EPS], "lam": LAMBDA})
    return out


CONFIGS = {"c1": c1, "c2": c2, "c3a": c3a, "c3b": c3b, "c5": c5}


# name: (file in the reference's data/ directory, numpy.loadtxt arguments, (n, d))
REAL = {
    "banknote": ("data_banknote_authentication.txt", {"delimiter": ",", "usecols": (0, 1, 2, 3)}, (1372, 4)),
    "yeast": ("yeast.data", {"usecols": (1, 2, 3, 4, 5, 6, 7, 8)}, (1484, 8)),
    "wilt": ("wilt.data", {"delimiter": ",", "usecols": (1, 2, 3, 4, 5)}, (4839, 5)),
    "ccpp": ("CCPP.data", {"delimiter": "\t", "skiprows": 1}, (9568, 5)),
    "eb": ("eb.arff", {"delimiter": ",", "usecols": (0, 1, 4)}, (45781, 3)),
    "skin_nonskin": ("Skin_NonSkin.txt", {"usecols": (0, 1, 2)}, (245057, 3)),
    "eeg_eye_state": ("EEG Eye State.arff", {"delimiter": ",", "usecols": tuple(range(14))}, (14980, 14)),
    "letter": ("letter-recognition.data", {"delimiter": ",", "usecols": tuple(range(1, 17))}, (20000, 16)),
    "iris": ("iris.data", {"delimiter": ","}, (150, 4)),
    "pendigits": ("pendigits.tra", {"delimiter": ","}, (7494, 17)),
}
REAL_EPS = 0.05


def load_real(name, data_dir):
    """One of the reference's real data sets from ``data_dir`` (a copy of its
    data/ directory), min-max normalised, float32 (python/data.py:44-103)."""
    f, kw, _ = REAL[name]
    return min_max_normalize(np.loadtxt(Path(data_dir) / f, **kw))


def stand_in(name, seed=0):
    """Seeded synthetic points with the shape of real data set ``name``."""
    n, d = REAL[name][2]
    rng = np.random.default_rng(seed)
    k = 8
    return blobs(rng, n, d, rng.uniform(0.2, 0.8, (k, d)), rng.uniform(0.02, 0.08, k), np.ones(k), 0.05)
