"""GPU min-max normalisation equals the reference's expression
(python/data.py:100-103) evaluated in float32, bit for bit."""
import numpy as np
import pytest

from eggsync import EggError, egg_sync, normalize

pytestmark = pytest.mark.gpu


def numpy_f32(X):
    X = X.astype(np.float32)
    lo, hi = X.min(0), X.max(0)
    span = (hi - lo).astype(np.float32)
    with np.errstate(invalid="ignore", divide="ignore"):
        out = ((X - lo).astype(np.float32) / span).astype(np.float32)
    return np.where(span > 0, out, np.float32(0)), lo, hi


@pytest.mark.parametrize("n,d", [(1, 3), (1000, 2), (300_001, 3), (5000, 17)])
def test_matches_numpy_float32(n, d):
    rng = np.random.default_rng(n + d)
    X = (rng.standard_normal((n, d)) * 7 + 3).astype(np.float32)
    X[:, 0] *= 100
    out, lo, hi = normalize(X)
    ref, rlo, rhi = numpy_f32(X)
    assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(lo, rlo) and np.array_equal(hi, rhi)


def test_device_in_place_and_clustering(gpu):
    import torch

    rng = np.random.default_rng(5)
    X = (rng.standard_normal((20000, 2)) * [3, 40] + [1, -7]).astype(np.float32)
    Xd = torch.from_numpy(X).to(gpu)
    normalize(Xd, out=Xd)
    ref, _, _ = numpy_f32(X)
    assert np.array_equal(Xd.cpu().numpy(), ref)
    a, _ = egg_sync(Xd, 0.05)
    b, _ = egg_sync(ref, 0.05)
    assert np.array_equal(a, b)


def test_constant_dimension_and_non_finite():
    X = np.ones((100, 2), np.float32)
    X[:, 1] = np.arange(100)
    out, lo, hi = normalize(X)
    assert np.all(out[:, 0] == 0) and out[-1, 1] == 1.0
    X[7, 0] = np.nan
    with pytest.raises(EggError) as e:
        normalize(X)
    assert e.value.status == -3
