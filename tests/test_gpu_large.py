"""GPU parity at the large workloads: 250k x 3 (eps 0.03), 500k x 3
(eps 0.02) and 1M x 3 (eps 0.015), seed 0.

* Along the loop's own trajectory: at iterations 0, 5, 20, 60, 120 and the
  last one, the positions the loop produces from the positions of the
  iteration before agree with the FP64 oracle's step from those positions
  on 4,000 sampled points (within 1e-5), the neighbour counts are exact, and
  a sampled point that violates the convergence rule clears the flag.  The
  positions come from runs capped at k and k + 1 iterations, so the step
  checked is the loop's incremental update (kept lanes, column masks,
  spanning-cell combines), not a fresh one.
* Against the reference EGG-SynC itself (fixtures ref_egg_<name>.npz made by
  tests/golden/make_golden_large.py; its three runs per workload gave one
  partition): the same iteration count, and the same partition up to a few
  disputed points.  Exact equality is not the bar at these sizes: the
  reference sums cells with float atomics in its own order, and over
  hundreds of iterations pairs of points sit within 1e-7 of eps (the float32
  rounding of their positions decides whether they are neighbours).  The
  FP64 oracle's own full runs disagree with the reference too: on the 500k
  workload in one point (and with this library in two, lying 4e-8 from a
  cell face), on the 250k workload in 9 points (and with this library in
  8; this library and the reference differ in 13); on
  the 1M workload 356 of the 387 disputed points are one collapsed group the
  reference merged with its neighbour after such a tie, while this library
  follows the FP64 oracle's step exactly for every one of them in all 191
  iterations.  The test bounds the disputed points at 0.05% of n.

Set EGG_PARITY_REPORT to a file path to append one JSON line per workload
with the largest coordinate error per checkpoint.
"""
import json
import os

import numpy as np
import pytest

from conftest import load_golden
from eggsync import data, egg_step, egg_sync
from make_golden import checksum
from oracle import ari

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5
LARGE = {"c3b_s0": data.c3b, "c2_s0": data.c2, "c5_s0": data.c5}
CHECKPOINTS = (0, 5, 20, 60, 120)
_cache = {}


def workload(name):
    if name not in _cache:
        c = LARGE[name](0)
        _cache[name] = (c["X"], c["eps"])
    return _cache[name]


def positions_after(X, eps, k):
    if k == 0:
        return X
    P = np.empty_like(X)
    egg_sync(X, eps, max_iter=k, positions_out=P)
    return P


@pytest.mark.parametrize("name", sorted(LARGE))
def test_large_trajectory_sampled(oracle, name):
    X, eps = workload(name)
    _, info = egg_sync(X, eps)
    T = info["iterations"]
    assert info["converged"] and T > 1
    ks = sorted({k for k in CHECKPOINTS if k < T} | {T - 1})
    idx = np.random.default_rng(1).choice(len(X), 4000, replace=False).astype(np.int32)
    errs = {}
    P = positions_after(X, eps, ks[0])
    for k in ks:
        P1 = positions_after(X, eps, k + 1)
        ox, ocnt, oviol = oracle.step_sample(P, eps, idx)
        err = float(np.abs(P1[idx] - ox).max())
        errs[k] = err
        assert err <= POS_TOL, "iteration %d: %.3g" % (k, err)
        _, cnt, flags = egg_step(P, eps)
        assert np.array_equal(cnt[idx], ocnt), "iteration %d" % k
        if oviol.any():
            assert flags[0] == 0, "iteration %d" % k
        nxt = [j for j in ks if j > k]
        P = P1 if nxt and nxt[0] == k + 1 else (positions_after(X, eps, nxt[0]) if nxt else None)
    rep = os.environ.get("EGG_PARITY_REPORT")
    if rep:
        with open(rep, "a") as f:
            f.write(json.dumps({"name": name, "n": len(X), "iterations": T, "max_abs_err": errs}) + "\n")


def disputed_points(a, b):
    """Points outside the largest overlap of their group in either labelling
    (-1 counts as one group)."""
    bad = np.zeros(len(a), bool)
    for A, B in ((a, b), (b, a)):
        key = A.astype(np.int64) * (int(B.max()) + 2) + (B.astype(np.int64) + 1)
        u, inv, cnt = np.unique(key, return_inverse=True, return_counts=True)
        la = u // (int(B.max()) + 2)
        best = {}
        for k, (g, c) in enumerate(zip(la, cnt)):
            if g not in best or c > best[g][1]:
                best[g] = (k, c)
        keep = np.zeros(len(u), bool)
        keep[[v[0] for v in best.values()]] = True
        bad |= ~keep[inv.ravel()]
    return np.flatnonzero(bad)


@pytest.mark.parametrize("name", sorted(LARGE))
def test_large_matches_reference_egg(name):
    """Against the reference EGG-SynC's own labels: the same iteration count,
    ARI >= 0.9999 and at most 0.05% disputed points (see the module
    docstring); or the recorded reason why the reference is undefined on
    this input."""
    G = load_golden("ref_egg_%s.npz" % name)
    X, eps = workload(name)
    assert checksum(X) == G["x_checksum"]
    if int(G["ref_ran"]) == 0:
        rows = G["pair_rows"]
        assert rows[:, 1].max() >= int(G["pair_limit"])
        pytest.skip(str(G["reason"]))
    lab, info = egg_sync(X, eps)
    ref = G["labels"][0]
    assert info["iterations"] == int(G["iterations"][0])
    assert ari(lab, ref) >= 0.9999
    assert len(disputed_points(lab, ref)) <= 5e-4 * len(X)
