"""CPU tests of the oracle: pinned against the reference's own code and
against the reference's formulas (no GPU needed)."""
import numpy as np
import pytest

from conftest import load_golden
from eggsync import data
from oracle import ari, same_partition


# geometry table computed from EGG_SynC.cu:1249-1260 for the benchmark configs
@pytest.mark.parametrize("n,d,eps,width,od,r", [
    (10_000, 2, 0.05, 56, 2, 3),
    (500_000, 3, 0.02, 173, 2, 4),
    (20_000, 16, 0.15, 53, 2, 8),
    (250_000, 3, 0.03, 115, 2, 4),
    (1_000_000, 3, 0.015, 230, 2, 4),
])
def test_geometry(oracle, n, d, eps, width, od, r):
    g = oracle.geometry(n, d, eps)
    assert g.width == width and g.od == od and g.r == r
    assert g.n_outer == width ** od
    assert abs(g.side - np.sqrt((eps / 2) ** 2 / d)) < 1e-8
    e = np.float32(eps)
    extra = np.float32(2 * e - np.float64(e) * np.sqrt(15 / 16) + np.float64(e) / 2 - np.sin(np.float64(e) / 2))
    assert g.eps_extra == extra


@pytest.mark.parametrize("e", [0.05, 0.02, 0.15, 0.015, 0.025, 1e-3])
def test_sq_threshold(oracle, e):
    e = np.float32(e)
    t = np.float32(oracle.sq_threshold(e))
    assert np.sqrt(t) <= e
    assert np.sqrt(np.nextafter(t, np.float32(np.inf))) > e


def test_step_matches_reference_sync_exact_box(oracle):
    """With the true box distance, the oracle's grid update equals the
    reference CPU SynC (SynC.cpp:16-40) run here: same neighbour counts up
    to distance ties at eps, same coordinates to 1e-6."""
    G = load_golden("ref_sync_c1.npz")
    c = data.c1(0)
    X, eps = c["X"], c["eps"]
    from make_golden import checksum  # noqa
    assert checksum(X) == G["x_checksum"]
    oracle.set_box_mode(True)
    try:
        Xn, cnt, _ = oracle.step(X, eps)
    finally:
        oracle.set_box_mode(False)
    same = cnt == G["counts"]
    assert (~same).sum() <= 3, "more than distance-tie mismatches"
    # mismatched points: the differing neighbour sits at |p - q| == eps up to rounding
    Xd = X.astype(np.float64)
    for p in np.nonzero(~same)[0]:
        dist = np.sqrt(((Xd - Xd[p]) ** 2).sum(1))
        assert np.any(np.abs(dist - eps) < 1e-6)
    assert np.abs(Xn[same] - G["step"][same]).max() <= 1e-6


def test_reference_egg_cell_test_differs_from_sync(oracle):
    """The reference EGG cell test (EGG_SynC.cu:613-636) is not exact: its
    "small" distance adds the nearer face also inside a cell's extent (drops
    neighbours), and the clamped last cell's box ends at width*side while its
    points reach 1.0 (may add neighbours).  The oracle reproduces both; extra
    neighbours only ever appear next to the upper edge."""
    G = load_golden("ref_sync_c1.npz")
    c = data.c1(0)
    X, eps = c["X"], c["eps"]
    _, cnt, _ = oracle.step(X, eps)
    assert (cnt < G["counts"]).sum() > 0
    more = np.nonzero(cnt > G["counts"])[0]
    g = oracle.geometry(len(X), X.shape[1], eps)
    edge = g.width * g.side
    assert np.all((X[more] > edge - 2 * eps).any(1))


def test_grid_vs_bruteforce(oracle):
    c = data.c1(1)
    X, eps = c["X"], c["eps"]
    oracle.set_box_mode(True)
    try:
        Xn, cnt, _ = oracle.step(X, eps)
    finally:
        oracle.set_box_mode(False)
    idx = np.arange(0, len(X), 7, dtype=np.int32)
    bx, bc = oracle.update_sample(X, eps, idx)
    same = bc == cnt[idx]
    assert (~same).sum() <= 1
    assert np.abs(bx[same] - Xn[idx][same]).max() <= 1e-6


def test_grid_structure(oracle):
    rng = np.random.default_rng(3)
    X = rng.random((3000, 3)).astype(np.float32)
    eps = 0.05
    order, cell_of, start = oracle.grid(X, eps)
    g = oracle.geometry(len(X), 3, eps)
    side = np.float32(g.side)
    ids = np.minimum((X / side).astype(np.int64), g.width - 1)
    outer = sum(ids[:, l] * g.width ** l for l in range(g.od))
    # within-cell order: Morton key of the top 2 bits of the in-cell offsets (d = 3)
    scale = np.float32(4) / side
    t = np.clip(((X - ids.astype(np.float32) * side) * scale).astype(np.int64), 0, 3)
    sub = np.zeros(len(X), np.int64)
    for k in (1, 0):
        for l in range(3):
            sub = (sub << 1) | ((t[:, l] >> k) & 1)
    key = [outer] + [ids[:, l] for l in range(g.od, 3)] + [sub]
    ref = np.lexsort(tuple([np.arange(len(X))] + key[::-1]))
    assert np.array_equal(order, ref)
    # every cell is a run of identical tuples, runs are maximal
    tup = ids[order]
    for c in range(len(start) - 1):
        seg = tup[start[c]:start[c + 1]]
        assert (seg == seg[0]).all()
        if c > 0:
            assert not (tup[start[c] - 1] == seg[0]).all()
    assert np.array_equal(cell_of[order], np.repeat(np.arange(len(start) - 1), np.diff(start)))


def test_labels_semantics(oracle):
    rng = np.random.default_rng(5)
    X = np.round(rng.random((500, 2)) * 20).astype(np.float32) / 20
    lab = oracle.labels(X, 0.05)
    order, cell_of, start = oracle.grid(X, 0.05)
    size = np.diff(start)[cell_of]
    assert np.array_equal(lab, np.where(size > 1, cell_of, -1))


def test_run_against_reference_egg_fixture(oracle):
    """Full-run labels of the oracle equal the reference EGG-SynC's run on a
    B200 (fixture), up to relabelling."""
    G = load_golden("ref_egg_c1_s0.npz")
    c = data.c1(0)
    lab, it, _, _ = oracle.run(c["X"], c["eps"])
    for k in range(len(G["labels"])):
        assert same_partition(lab, G["labels"][k])
    assert it == int(G["iterations"][0])


def test_ari():
    a = np.array([0, 0, 1, 1, -1, -1])
    assert ari(a, a) == 1.0
    assert ari(a, np.array([5, 5, 3, 3, -1, -1])) == 1.0
    assert ari(a, np.array([0, 1, 0, 1, -1, -1])) < 1.0
    assert same_partition(a, np.array([7, 7, 2, 2, -1, -1]))
    assert not same_partition(a, np.array([7, 7, 7, 2, -1, -1]))


def test_extra_check_detects_pull(oracle):
    """p and q just beyond eps, with a point of q's eps/2 group inside the
    eps-ball of p: the extra check (EGG_SynC.cu:1037-1203) must veto."""
    eps = np.float32(0.05)
    p = np.array([0.30, 0.50], np.float32)
    q = np.array([0.30 + 1.01 * 0.05, 0.50], np.float32)
    r = np.array([q[0] - 0.02, 0.50], np.float32)   # within eps/2 of q, within eps of p
    X = np.stack([p, q, r])
    ok, pairs = oracle.extra_check(X, eps)
    assert pairs >= 1 and ok == 0
    # without r the MBR of q is q itself, outside eps: converged
    ok2, pairs2 = oracle.extra_check(np.stack([p, q]), eps)
    assert pairs2 >= 1 and ok2 == 1


def test_ref_annulus_pairs_equals_walked_count(oracle):
    """The reference's extra-check pair count (EGG_SynC.cu:767-878), counted
    with tight-box shortcuts, equals the count of the oracle's plain walk
    over the same cells on converged input (no veto, so every pair is
    walked), and the 2-D layout of five tight clusters 0.051 apart (inside
    the (eps, eps_extra] annulus of their neighbours) bounds it."""
    rng = np.random.default_rng(5)
    eps = np.float32(0.05)
    X = np.concatenate([np.array([0.2 + 0.051 * k, 0.5]) + rng.uniform(-1e-4, 1e-4, (40, 2)) for k in range(5)])
    X = X.astype(np.float32)
    ok, walked = oracle.extra_check(X, eps)
    total, worst = oracle.ref_annulus_pairs(X, eps)
    assert ok == 1
    assert total == walked
    assert 0 < total <= 2 * 4 * 40 * 40
    assert 0 < worst <= 80


@pytest.mark.parametrize("name", ["c3b_s0", "c2_s0", "c5_s0"])
def test_large_reference_fixtures(name):
    """The reference EGG-SynC fixtures of the large workloads: made from the
    same inputs, the reference's pair count stayed inside its int limits, and
    its repeated runs gave one partition and one iteration count."""
    from make_golden import checksum
    from oracle import ref_egg_pair_limit

    G = load_golden("ref_egg_%s.npz" % name)
    X = {"c3b_s0": data.c3b, "c2_s0": data.c2, "c5_s0": data.c5}[name](0)["X"]
    assert checksum(X) == G["x_checksum"]
    assert int(G["ref_ran"]) == 1 and int(G["ref_runs_same_partition"]) == 1
    assert G["pair_rows"][:, 1].max() < ref_egg_pair_limit(len(X)) == int(G["pair_limit"])
    assert len(set(G["iterations"].tolist())) == 1
    assert G["labels"].shape == (1, len(X))


def test_disputed_points_counts_only_the_minority():
    from test_gpu_large import disputed_points

    a = np.array([0, 0, 0, 1, 1, 1, -1, -1], np.int32)
    b = np.array([5, 5, 7, 2, 2, 2, -1, 3], np.int32)
    assert disputed_points(a, b).tolist() == [2, 7]
    assert len(disputed_points(a, a)) == 0
