"""Error paths on the host, without a GPU fault: an allocation failure
injected through egg_inject_alloc_failures (the next k device allocations
fail as cudaMalloc does on an exhausted device, nothing is allocated) must
come back as EGG_ERR_CUDA with a message, and the next call must allocate
again and give the normal result (the reference exits the process on any
CUDA error, EGG_SynC.cu:20-26)."""
import numpy as np
import pytest

from eggsync import EggError, _lib, data, egg_sync, egg_sync_batch, normalize, simple_sync

pytestmark = pytest.mark.gpu


def _expect_cuda_error(fn):
    with pytest.raises(EggError) as e:
        fn()
    assert e.value.status == _lib.EGG_ERR_CUDA
    assert "out of memory" in str(e.value).lower() or "memory" in str(e.value).lower()


def test_sync_run_recovers_after_failed_workspace_allocation(eggsync_lib):
    L = eggsync_lib
    c = data.c1(0)
    ref, ri = egg_sync(c["X"], c["eps"])
    assert L.egg_release() == _lib.EGG_OK  # the next call must allocate its workspace
    assert L.egg_inject_alloc_failures(1) == _lib.EGG_OK
    _expect_cuda_error(lambda: egg_sync(c["X"], c["eps"]))
    lab, info = egg_sync(c["X"], c["eps"])  # allocates again
    assert np.array_equal(lab, ref) and info["iterations"] == ri["iterations"]


def test_batch_and_brute_force_paths_recover(eggsync_lib):
    L = eggsync_lib
    X = data.c1(1)["X"][:3000]
    inst = [(X, 0.05), (X, 0.04)]
    ref = egg_sync_batch(inst)[0]
    assert L.egg_release() == _lib.EGG_OK
    assert L.egg_inject_alloc_failures(1) == _lib.EGG_OK
    _expect_cuda_error(lambda: egg_sync_batch(inst))
    got = egg_sync_batch(inst)[0]
    assert all(np.array_equal(a[0], b[0]) for a, b in zip(ref, got))
    sref, _ = simple_sync(X[:800], 0.05)
    assert L.egg_inject_alloc_failures(1) == _lib.EGG_OK
    _expect_cuda_error(lambda: simple_sync(X[:800], 0.05))
    s2, _ = simple_sync(X[:800], 0.05)
    assert np.array_equal(sref, s2)
    assert L.egg_inject_alloc_failures(0) == _lib.EGG_OK


def test_normalize_recovers(eggsync_lib):
    L = eggsync_lib
    raw = np.random.default_rng(2).normal(0, 3, (5000, 3)).astype(np.float32)
    ref = normalize(raw)  # (normalised points, minima, maxima)
    assert L.egg_inject_alloc_failures(1) == _lib.EGG_OK
    _expect_cuda_error(lambda: normalize(raw))
    got = normalize(raw)
    assert all(np.array_equal(a, b) for a, b in zip(got, ref))
