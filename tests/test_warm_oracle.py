"""CPU checks of the warm-start oracle (oracle/mlp_oracle.py): its gradient
against central finite differences, its feature layout on a hand-checked
case, and its BF16 rounding."""
import numpy as np

import mlp_oracle as M


def small_model(d, seed=0):
    rng = np.random.default_rng(seed)
    F, H = M.feature_dim(d), 128
    return {"w1": rng.standard_normal((F, H)) * 0.1, "b1": rng.standard_normal(H) * 0.1,
            "w2": rng.standard_normal((H, H)) * 0.1, "b2": rng.standard_normal(H) * 0.1,
            "w3": rng.standard_normal((H, d)) * 0.1, "b3": rng.standard_normal(d) * 0.1}


def test_gradient_matches_finite_differences():
    d = 2
    rng = np.random.default_rng(1)
    w = small_model(d)
    x = rng.standard_normal((7, M.feature_width(d)))
    t = rng.standard_normal((7, d))
    loss, g = M.grad(w, x, t, d)
    assert abs(loss - M.mse(w, x, t, d)) < 1e-12
    h = 1e-6
    for name in M.NAMES:
        flat = w[name].reshape(-1)
        for idx in rng.choice(flat.size, min(6, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp = M.mse(w, x, t, d)
            flat[idx] = old - h
            lm = M.mse(w, x, t, d)
            flat[idx] = old
            num = (lp - lm) / (2 * h)
            assert abs(num - g[name].reshape(-1)[idx]) <= 1e-6 + 1e-5 * abs(num), name


def test_feature_layout_two_points():
    # two points in one coarse cell of a 1-D grid (eps 0.25: 4 cells)
    X = np.array([[0.30], [0.45]], np.float32)
    f = M.features(X, 0.25)
    assert f.shape == (2, 16) and M.feature_dim(1) == 10
    # offsets in the cell: 0.2 and 0.8
    assert np.allclose(f[:, 0], [0.2, 0.8], atol=1e-6)
    # neighbour -1 (cell 0) is empty, neighbour 0 holds both points, +1 empty
    assert np.all(f[:, 1:4] == 0) and np.all(f[:, 7:10] == 0)
    assert np.allclose(f[:, 4], np.log1p(2) / 8, atol=1e-7)
    # centroid (0.5) minus point, spread 0.3
    assert np.allclose(f[:, 5], [0.3, -0.3], atol=1e-6)
    assert np.allclose(f[:, 6], [0.3, 0.3], atol=1e-6)
    assert np.all(f[:, 10:] == 0)


def test_bf16_rounding():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0], np.float32)
    r = M.bf16(a)
    assert r[0] == 1.0
    assert r[1] == 1.0  # halfway between 1 and 1 + 2^-7: ties to even
    assert r[2] == 1.0 + 2 ** -7  # nearer to the next bf16
    assert r[3] == -2.5 and r[4] == 0.0
