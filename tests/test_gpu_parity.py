"""GPU parity tests: the CUDA path (through the C ABI) against the oracle
and against the reference EGG-SynC's own results (fixtures).

Bars: grid, counts, flags and labels are bit-exact (integer work); positions
within 1e-5 absolute of the FP64 oracle per iteration (coordinates are
min-max normalised to [0, 1])."""
import numpy as np
import pytest

from conftest import load_golden
from eggsync import EggError, data, egg_grid, egg_step, egg_sync
from make_golden import checksum, small_cases
from oracle import ari, same_partition

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5


def cases():
    out = {"c1_s0": (data.c1(0)["X"], 0.05), "c1_s1": (data.c1(1)["X"], 0.05), "c3a_s0": (data.c3a(0)["X"], 0.15)}
    out.update(small_cases())
    return out


CASES = cases()
NAMES = sorted(CASES)


@pytest.mark.parametrize("name", NAMES)
def test_grid_matches_oracle(oracle, name):
    X, eps = CASES[name]
    order, cell_of, start = egg_grid(X, eps)
    o_order, o_cell_of, o_start = oracle.grid(X, eps)
    assert np.array_equal(order, o_order)
    assert np.array_equal(start, o_start)
    assert np.array_equal(cell_of, o_cell_of[o_order])


@pytest.mark.parametrize("name", NAMES)
def test_step_matches_oracle(oracle, name):
    X, eps = CASES[name]
    xn, cnt, flags = egg_step(X, eps)
    oxn, ocnt, oflag = oracle.step(X, eps)
    assert np.array_equal(cnt, ocnt)
    assert flags[0] == oflag
    assert np.abs(xn - oxn).max() <= POS_TOL
    if oflag:
        ok, _ = oracle.extra_check(X, eps)
        assert flags[1] == ok
    else:
        assert flags[1] == 0


@pytest.mark.parametrize("name", ["c1_s0", "c3a_s0", "borders", "duplicates", "d1", "n300"])
def test_trajectory_per_iteration(oracle, name):
    """Every iteration of the GPU loop, from the GPU's own positions: the
    oracle step from the same positions agrees (counts and flags exactly,
    positions within 1e-5)."""
    X, eps = CASES[name]
    x = X
    worst = 0.0
    for it in range(200):
        xn, cnt, flags = egg_step(x, eps)
        oxn, ocnt, oflag = oracle.step(x, eps)
        assert np.array_equal(cnt, ocnt), "iteration %d" % it
        assert flags[0] == oflag, "iteration %d" % it
        worst = max(worst, float(np.abs(xn - oxn).max()))
        assert worst <= POS_TOL, "iteration %d" % it
        if flags[0]:
            ok, _ = oracle.extra_check(x, eps)
            assert flags[1] == ok
        if flags[1]:
            break
        x = xn
    else:
        pytest.fail("no convergence in 200 iterations")


@pytest.mark.parametrize("name", NAMES)
def test_run_matches_oracle(oracle, name):
    X, eps = CASES[name]
    lab, info = egg_sync(X, eps)
    olab, oit, _, _ = oracle.run(X, eps)
    assert info["converged"]
    assert info["iterations"] == oit
    assert same_partition(lab, olab)
    assert np.array_equal(lab, olab)  # same cell numbering as the oracle's grid order


@pytest.mark.parametrize("name", NAMES)
def test_run_matches_reference_egg(name):
    """ARI = 1 against the reference EGG-SynC's own labels on the same input."""
    G = load_golden("ref_egg_%s.npz" % name)
    X, eps = CASES[name]
    assert checksum(X) == G["x_checksum"]
    lab, info = egg_sync(X, eps)
    for k in range(len(G["labels"])):
        assert ari(lab, G["labels"][k]) == 1.0
    assert info["iterations"] == int(G["iterations"][0])


@pytest.mark.parametrize("name", ["c1_s0", "c3a_s0", "noise", "d5", "borders"])
def test_incremental_equals_full_update(name):
    """Reusing the results of points whose stencil region did not change is
    bit-identical to recomputing every point in every iteration."""
    X, eps = CASES[name]
    pa = np.empty_like(X)
    pb = np.empty_like(X)
    la, ia = egg_sync(X, eps, positions_out=pa)
    lb, ib = egg_sync(X, eps, full_update=True, positions_out=pb)
    assert ia["iterations"] == ib["iterations"]
    assert np.array_equal(la, lb)
    assert np.array_equal(pa.view(np.uint32), pb.view(np.uint32))


@pytest.mark.parametrize("name", ["c1_s0", "c3a_s0", "duplicates", "noise", "d1"])
def test_union_find_labels_equal_cell_labels(name):
    """GPU union-find cluster extraction gives the reference's partition and
    label values (the direct per-cell labelling)."""
    X, eps = CASES[name]
    a, ia = egg_sync(X, eps)  # union-find (default)
    b, ib = egg_sync(X, eps, labels_mode="cells")
    assert np.array_equal(a, b)
    assert ia["n_clusters"] == ib["n_clusters"] == len(np.unique(a[a >= 0]))


@pytest.mark.parametrize("name", ["c1_s0", "c3a_s0", "noise", "d5"])
def test_order_parameter_bounds_contain_exact(oracle, name):
    """The certified FP64 interval of the local order parameter contains the
    exact value over the same neighbourhoods (oracle), on the input and on
    the final positions."""
    X, eps = CASES[name]
    # of the input: one iteration with the every-iteration mode
    _, info = egg_sync(X, eps, max_iter=1, order_param=2)
    lo, hi = info["itr_order_param"][0]
    exact = oracle.order_parameter_egg(X, eps)
    assert lo <= exact <= hi and hi - lo < 0.05
    # of the final positions
    P = np.empty_like(X)
    lab, info = egg_sync(X, eps, order_param=1, positions_out=P)
    lo, hi = info["order_param"]
    exact = oracle.order_parameter_egg(P, eps)
    assert lo <= exact <= hi
    assert hi - lo < 1e-4  # collapsed clusters: the interval is tight
    # reporting does not change the run
    lab2, info2 = egg_sync(X, eps)
    assert np.array_equal(lab, lab2) and info2["iterations"] == info["iterations"]


def test_lambda_stop_rule():
    """stop_rule="lambda" stops at the first iteration whose certified lower
    bound reaches lambda (SynC.cpp:277-303 semantics on the EGG neighbourhoods)."""
    X, eps = CASES["c1_s0"]
    lab, info = egg_sync(X, eps, lam=0.999, stop_rule="lambda")
    r = info["itr_order_param"]
    assert info["converged"] and len(r) == info["iterations"]
    assert r[-1][0] >= 0.999
    assert all(lo < 0.999 for lo, _ in r[:-1])
    assert all(lo <= hi for lo, hi in r)


def test_deterministic_and_loop_modes():
    X, eps = CASES["c1_s0"]
    a, ia = egg_sync(X, eps)
    b, ib = egg_sync(X, eps)
    c, ic = egg_sync(X, eps, loop="host")
    assert np.array_equal(a, b) and np.array_equal(a, c)
    assert ia["iterations"] == ib["iterations"] == ic["iterations"]
    x1, _, _ = egg_step(X, eps)
    x2, _, _ = egg_step(X, eps)
    assert np.array_equal(x1.view(np.uint32), x2.view(np.uint32))


def test_device_tensors(gpu):
    import torch

    X, eps = CASES["c1_s0"]
    a, _ = egg_sync(X, eps)
    Xd = torch.from_numpy(X).to(gpu)
    out = torch.empty(len(X), dtype=torch.int32, device=gpu)
    b, _ = egg_sync(Xd, eps, labels_out=out)
    assert np.array_equal(a, b.cpu().numpy())


def test_drop_in_wrapper():
    import torch
    from eggsync import EGG_SynC

    X, eps = CASES["c1_s0"]
    C, itr_times, stage_times, space = EGG_SynC(torch.from_numpy(X), eps)
    lab, info = egg_sync(X, eps)
    assert C.dtype == torch.float32 and C.shape == (len(X),)
    assert np.array_equal(C.numpy().astype(np.int32), lab)
    assert itr_times.shape == (info["iterations"],)
    assert stage_times.shape == (6,) and space.dtype == torch.int32


def test_edge_cases(oracle):
    # one point
    lab, info = egg_sync(np.array([[0.5, 0.5]], np.float32), 0.05)
    assert lab.tolist() == [-1] and info["iterations"] == 1
    # identical points: one cluster after one iteration
    X = np.full((100, 3), 0.25, np.float32)
    lab, info = egg_sync(X, 0.05)
    assert (lab == lab[0]).all() and lab[0] >= 0 and info["iterations"] == 1
    # n < cells per dimension: no outer grid dimension (the reference is undefined here)
    X = np.array([[0.1, 0.1], [0.12, 0.1], [0.9, 0.9]], np.float32)
    lab, info = egg_sync(X, 0.05)
    olab, oit, _, _ = oracle.run(X, 0.05)
    assert np.array_equal(lab, olab) and info["iterations"] == oit
    # non-finite input
    X = np.random.default_rng(0).random((50, 2)).astype(np.float32)
    X[3, 1] = np.nan
    with pytest.raises(EggError) as e:
        egg_sync(X, 0.05)
    assert e.value.status == -3


def test_large_sampled_step(oracle):
    """500k x 3 (c2): the first iteration of 4,000 sampled points equals the
    oracle's exactly in counts and to 1e-5 in position."""
    c = data.c2(0)
    X, eps = c["X"], c["eps"]
    xn, cnt, flags = egg_step(X, eps)
    idx = np.random.default_rng(1).choice(len(X), 4000, replace=False).astype(np.int32)
    oxs, ocnt, oviol = oracle.step_sample(X, eps, idx)
    assert np.array_equal(cnt[idx], ocnt)
    assert np.abs(xn[idx] - oxs).max() <= POS_TOL
    assert flags[0] == 0 and oviol.any()


def test_large_run_properties():
    """1M x 3 (c5 shape): converges; every label is a set of points sharing
    one final cell; a second run is identical."""
    c = data.c5(0)
    X, eps = c["X"], c["eps"]
    pa = np.empty_like(X)
    lab, info = egg_sync(X, eps, positions_out=pa)
    assert info["converged"] and info["iterations"] > 1
    assert info["n_clusters"] == len(np.unique(lab[lab >= 0]))
    # the labels are exactly the final grid's cells holding > 1 point
    order, cell_of, start = egg_grid(pa, eps)
    size = np.diff(start)[cell_of]
    lab_sorted = np.where(size > 1, cell_of, -1)
    assert np.array_equal(lab[order], lab_sorted)
    # a second run, and a run that recomputes every point every iteration,
    # give the same bits
    pb = np.empty_like(X)
    lab2, info2 = egg_sync(X, eps, full_update=True, positions_out=pb)
    assert np.array_equal(lab, lab2) and info2["iterations"] == info["iterations"]
    assert np.array_equal(pa.view(np.uint32), pb.view(np.uint32))
