"""The update stencil's column screen never drops a cell the reference's box
test can pass.

The host keeps an outer column (offsets k_0..k_{od-1}) only when
a = sum_l ((|k_l| - 1.001)+)^2 <= R2 = t_eps / side^2 * (1 + 1e-3).  Here the
reference's "small" box distance (EGG_SynC.cu:613-636, with the fused face
offsets the CUDA kernels and the oracle use) is evaluated in float32 for
random points against every cell offset within r + 1, and every cell that
passes must lie in a kept column.  The same bound also limits the offset in
the next dimension, which the test checks as a sanity bound on the screen's
arithmetic.
"""
import numpy as np
import pytest


def f32_fma(a, b, c):
    # a * b + c rounded once to float32: the product of two float32 values is
    # exact in float64, and so is the sum here (the magnitudes are close)
    return np.float32(np.float64(a) * np.float64(b) + np.float64(c))


def sq_threshold(e):
    e = np.float32(e)
    t = np.float32(e * e)
    while t > 0 and np.sqrt(t) > e:
        t = np.nextafter(t, np.float32(0))
    while np.sqrt(np.nextafter(t, np.float32(np.inf))) <= e:
        t = np.nextafter(t, np.float32(np.inf))
    return t


def small_box(x, cd, side):
    s = np.float32(0)
    for xl, c in zip(x, cd):
        left = f32_fma(np.float32(c), side, -xl)
        right = f32_fma(np.float32(c + 1), side, -xl)
        left = np.float32(left * left)
        right = np.float32(right * right)
        s = np.float32(s + (left if left < right else right))
    return s


@pytest.mark.parametrize("d,eps,od", [(2, 0.05, 2), (3, 0.015, 2), (3, 0.03, 2), (5, 0.08, 2)])
def test_screen_keeps_every_passing_cell(d, eps, od):
    side = np.float32(np.sqrt((eps / 2) ** 2 / d))
    width = int(np.float32(1) / side)
    r = int(np.ceil(np.float32(eps) / side))
    t = sq_threshold(eps)
    R2 = float(t) / (float(side) * float(side)) * (1 + 1e-3)

    def excess(k):
        v = abs(k) - 1.001
        return v * v if v > 0 else 0.0

    rng = np.random.default_rng(d)
    rad = r + 1
    offs = np.array(np.meshgrid(*[np.arange(-rad, rad + 1)] * min(d, 3), indexing="ij")).reshape(min(d, 3), -1).T
    passed = 0
    for _ in range(60):
        gi = rng.integers(rad, width - rad, d)
        x = ((gi + rng.random(d)) * side).astype(np.float32)
        x = np.where(rng.random(d) < 0.2, (gi * side).astype(np.float32), x)  # points on faces too
        gi = np.array([min(int(np.float32(xl) / side), width - 1) for xl in x])
        for k in offs:
            kk = np.zeros(d, int)
            kk[: len(k)] = k
            if small_box(x, gi + kk, side) > t:
                continue
            passed += 1
            a = sum(excess(v) for v in kk[:od])
            assert a <= R2, (kk, a, R2)
            if od < d:
                assert excess(kk[od]) <= R2 - a, (kk, a)
    assert passed > 0
