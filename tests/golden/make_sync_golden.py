"""Golden record of the reference's full SynC eps search, Sync(D, k)
(python/SynCTorch.py:349-372), on the four small inputs of ref_mdl.npz.

Sync starts at eps = NN(k), grows it by NN(k + 1) - NN(k), clusters every
eps with the Python SynC (DynamicalClustering + synCluster,
SynCTorch.py:64-95, 317-346: neighbours at distance < eps, stop once the mean
local order parameter exceeds lam, clusters = groups of allclose points) and
keeps the clustering of least L_Clust_Outl cost.  DynamicalClustering calls
its callback unconditionally (SynCTorch.py:320), so a no-op callback is
passed; `double` is supplied as `float` as in make_mdl_golden.py.  Stored
per input: the eps schedule, the cluster count and cost of every
candidate, the index picked, and the picked clusters as labels.

    python tests/golden/make_sync_golden.py REFERENCE_TREE   (k = 5)
"""
import contextlib
import io
import os
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import make_mdl_golden as mg  # noqa: E402  (reads the reference tree from argv / EGG_REFERENCE_ROOT)

K = 5


def main():
    ref = mg.load_ref()
    res = {}
    for name, X, _labels in mg.cases():
        D = torch.from_numpy(X)
        Ms, costs, eps_list = [], [], []
        eps = ref.NN(K, D)
        delta = ref.NN(K + 1, D) - eps
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            while True:
                eps_list.append(float(eps))
                M = ref.DynamicalClustering(D, eps, call=lambda _d: None)
                Ms.append(M)
                costs.append(float(ref.L_Clust_Outl(D, M)))
                eps += delta
                if len(M[0]) == 1:
                    break
        best = int(torch.argmin(torch.DoubleTensor(costs)))
        lab = np.full(len(X), -1, np.int32)
        for c, members in enumerate(Ms[best][0]):
            lab[np.array(members, np.int64)] = c
        res[name + "_eps"] = np.array(eps_list, np.float64)
        res[name + "_nclusters"] = np.array([len(M[0]) for M in Ms], np.int32)
        res[name + "_costs"] = np.array(costs, np.float64)
        res[name + "_best"] = np.int32(best)
        res[name + "_labels"] = lab
        print(name, "candidates", len(costs), "best", best, "clusters", [len(M[0]) for M in Ms], flush=True)
    np.savez(HERE / "ref_sync_search.npz", k=np.int32(K), **res)


if __name__ == "__main__":
    main()
