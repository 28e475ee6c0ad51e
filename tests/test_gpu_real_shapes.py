"""EGG-SynC on seeded stand-ins with the shapes of the reference's real data
sets (eggsync.data.REAL: n 150-245,057, d 3-17), at the experiments' eps
0.05 (run_experiment.py:12, 547-551).

Up to 20,000 points the whole run is checked against the oracle (same
iteration count, same labels); the two larger shapes through the
size-independent properties: a repeated run and a run recomputing every
point give the same bits, the per-cell labelling equals the union-find one."""
import numpy as np
import pytest

from eggsync import data, egg_sync

pytestmark = pytest.mark.gpu

SMALL = [k for k, v in data.REAL.items() if v[2][0] <= 20_000]
LARGE = [k for k, v in data.REAL.items() if v[2][0] > 20_000]


@pytest.mark.parametrize("name", SMALL)
def test_stand_in_matches_oracle(oracle, name):
    X = data.stand_in(name)
    lab, info = egg_sync(X, data.REAL_EPS)
    olab, oit, _, _ = oracle.run(X, data.REAL_EPS)
    assert info["converged"]
    assert info["iterations"] == oit
    assert np.array_equal(lab, olab)


@pytest.mark.parametrize("name", LARGE)
def test_stand_in_properties(name):
    X = data.stand_in(name)
    P1, P2 = np.empty_like(X), np.empty_like(X)
    lab, info = egg_sync(X, data.REAL_EPS, positions_out=P1)
    assert info["converged"] and info["n_clusters"] >= 1
    lab2, info2 = egg_sync(X, data.REAL_EPS, positions_out=P2, full_update=True)
    assert info2["iterations"] == info["iterations"]
    assert np.array_equal(lab, lab2) and np.array_equal(P1.view(np.uint32), P2.view(np.uint32))
    lab3, _ = egg_sync(X, data.REAL_EPS, labels_mode="cells")
    assert np.array_equal(lab, lab3)
