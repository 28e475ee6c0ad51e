"""The MDL eps-search oracle against the reference's own functions (CPU).

tests/golden/ref_mdl.npz holds NN(k, D) and L_Clust_Outl(D, M) of
python/SynCTorch.py computed on small seeded inputs
(tests/golden/make_mdl_golden.py).  The reference computes in float32, the
oracle in float64: NN agrees to 1e-6 relative, the cost to 1e-7."""
import numpy as np
import pytest

from conftest import GOLDEN
import mdl_oracle as M

REF = np.load(GOLDEN / "ref_mdl.npz")
NAMES = ("s0", "s1", "s2", "s3")


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("k", (1, 2, 3, 5))
def test_nn_mean_matches_reference(name, k):
    X = REF[name + "_X"]
    assert M.nn_mean(X, k) == pytest.approx(float(REF["%s_nn%d" % (name, k)]), rel=1e-6)


@pytest.mark.parametrize("name", NAMES)
def test_cost_matches_reference(name):
    X, lab = REF[name + "_X"], REF[name + "_labels"]
    assert (lab == -1).any() and len(M.clusters_of(lab)) > 1  # outliers and several clusters covered
    assert M.mdl_cost(X, lab) == pytest.approx(float(REF[name + "_cost"]), rel=1e-7)


def test_cost_ignores_label_values_and_order():
    X, lab = REF["s1_X"], REF["s1_labels"]
    remap = np.where(lab >= 0, 1000 - lab, -1)
    assert M.mdl_cost(X, remap) == pytest.approx(M.mdl_cost(X, lab), rel=1e-12)


def test_eps_schedule_is_float32():
    eps, step = M.eps_schedule(0.1, 0.13, 5)
    assert eps.dtype == np.float32 and step.dtype == np.float32
    e = np.float32(0.1)
    for v in eps:
        assert v == e
        e = np.float32(e + (np.float32(0.13) - np.float32(0.1)))


def test_search_stops_at_one_cluster_and_takes_first_minimum():
    X = REF["s0_X"]
    n = len(X)
    calls = []

    def cluster(eps):
        calls.append(eps)
        c = len(calls)
        if c >= 4:
            return np.zeros(n, np.int32)  # one cluster: the search ends here
        return (np.arange(n) % (5 - c)).astype(np.int32)

    best, costs, eps, ks = M.search(X, 3, cluster, max_candidates=50)
    assert len(calls) == 4 and ks[-1] == 1 and list(ks[:-1]) == [4, 3, 2]
    assert best == int(np.argmin(costs))
    assert eps[0] == np.float32(M.nn_mean(X, 3))
