"""Golden vectors of the MDL eps search pieces from the reference's own code.

Runs NN(k, D) and L_Clust_Outl(D, M) of python/SynCTorch.py (the reference
tree is the first argument, or EGG_REFERENCE_ROOT) on small seeded inputs and writes
tests/golden/ref_mdl.npz.  The reference module uses ``double('inf')``
without defining ``double``; the generator supplies ``double = float``
(the only change) so that NN runs as written.

    python tests/golden/make_mdl_golden.py REFERENCE_TREE
"""
import contextlib
import importlib.util
import io
import sys
from pathlib import Path

import numpy as np
import scipy.stats  # noqa: F401  (the reference reaches scipy.stats.iqr through `import scipy`)
import torch

HERE = Path(__file__).resolve().parent
import os

_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EGG_REFERENCE_ROOT")
if not _root:
    sys.exit("usage: make_mdl_golden.py REFERENCE_TREE (or set EGG_REFERENCE_ROOT)")
REF = Path(_root)


def load_ref():
    spec = importlib.util.spec_from_file_location("ref_synctorch", REF / "python" / "SynCTorch.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.double = float
    return mod


def cases():
    """(name, X float32, labels): blobs with a few outliers, labels from a
    coarse grid (cells with one point are outliers)."""
    out = []
    for seed, n, d, cell in ((0, 60, 2, 0.25), (1, 90, 3, 0.34), (2, 70, 2, 0.5), (3, 50, 4, 0.5)):
        rng = np.random.default_rng(seed)
        k = 3
        centres = rng.uniform(0.2, 0.8, (k, d))
        X = centres[rng.integers(0, k, n)] + rng.normal(0, 0.06, (n, d))
        X[: n // 10] = rng.uniform(0, 1, (n // 10, d))
        X = ((X - X.min(0)) / (X.max(0) - X.min(0))).astype(np.float32)
        key = np.floor(X / cell).astype(np.int64) @ (1000 ** np.arange(d))
        _, inv, cnt = np.unique(key, return_inverse=True, return_counts=True)
        labels = np.where(cnt[inv] > 1, inv, -1).astype(np.int32)
        out.append(("s%d" % seed, X, labels))
    return out


def main():
    ref = load_ref()
    res = {}
    for name, X, labels in cases():
        D = torch.from_numpy(X)
        for k in (1, 2, 3, 5):
            res["%s_nn%d" % (name, k)] = np.float64(ref.NN(k, D))
        C = [list(np.nonzero(labels == c)[0]) for c in np.unique(labels[labels >= 0])]
        with contextlib.redirect_stdout(io.StringIO()):
            cost = ref.L_Clust_Outl(D, (C, []))
        res[name + "_X"] = X
        res[name + "_labels"] = labels
        res[name + "_cost"] = np.float64(cost)
    np.savez(HERE / "ref_mdl.npz", **res)
    print("wrote", HERE / "ref_mdl.npz", len(res), "arrays")


if __name__ == "__main__":
    main()
