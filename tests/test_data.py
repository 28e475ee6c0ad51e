import numpy as np

from eggsync import data


def test_generators_are_seeded_and_normalised():
    for name in ("c1", "c3a"):
        a = data.CONFIGS[name](0)
        b = data.CONFIGS[name](0)
        c = data.CONFIGS[name](1)
        assert np.array_equal(a["X"], b["X"])
        assert not np.array_equal(a["X"], c["X"])
        X = a["X"]
        assert X.dtype == np.float32 and X.flags.c_contiguous
        assert X.min() == 0.0 and X.max() == 1.0
        assert np.all(X.min(0) == 0) and np.all(X.max(0) == 1)


def test_shapes():
    assert data.c1(0)["X"].shape == (10_000, 2)
    assert data.c3a(0)["X"].shape == (20_000, 16)
    inst = data.c4(0, instances=4)
    for it in inst:
        n, d = it["X"].shape
        assert 1_000 <= n <= 200_000 and d in (2, 3, 5)
        assert len(it["eps"]) == 8
    assert abs(data.C4_EPS[0] - 0.01) < 1e-6 and abs(data.C4_EPS[-1] - 0.08) < 1e-6


def test_min_max_normalize_matches_reference_formula():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(100, 3)) * 50
    ref = (X - X.min(0)) / (X.max(0) - X.min(0))
    assert np.allclose(data.min_max_normalize(X), ref.astype(np.float32))


def test_load_real_reads_the_reference_formats(tmp_path):
    """Files in each real data set's layout (columns, delimiter, header) give
    the configured columns, min-max normalised."""
    rng = np.random.default_rng(5)
    for name, (fname, kw, (n, d)) in data.REAL.items():
        cols = max(kw.get("usecols", (d - 1,))) + 1 if "usecols" in kw else d
        V = rng.uniform(-5, 5, (7, cols))
        delim = kw.get("delimiter", " ")
        lines = [delim.join("%.6f" % v for v in row) for row in V]
        if kw.get("skiprows"):
            lines = ["header"] * kw["skiprows"] + lines
        (tmp_path / fname).write_text("\n".join(lines) + "\n")
        X = data.load_real(name, tmp_path)
        want = V[:, list(kw["usecols"])] if "usecols" in kw else V
        assert X.shape == (7, d) and X.dtype == np.float32
        np.testing.assert_allclose(X, (want - want.min(0)) / (want.max(0) - want.min(0)), atol=1e-6)


def test_stand_ins_have_the_real_shapes():
    for name, (_, _, shape) in data.REAL.items():
        if shape[0] > 50_000:
            continue
        X = data.stand_in(name)
        assert X.shape == shape and X.dtype == np.float32
        assert X.min() >= 0 and X.max() <= 1
        assert np.array_equal(X, data.stand_in(name))
