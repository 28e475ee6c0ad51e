"""The allocation-free grid build, egg_sync_grid_noalloc, called through the C ABI.

It exists for callers that must not allocate device memory (a host framework
that owns the device through its own memory pool, or a caller that cannot
afford the device synchronisation of cudaMalloc/cudaFree).  Its results must
be those of the ordinary entry point, egg_sync_grid, which uses the
library's allocated workspace.  This file is collected last so that, if it
fails, a run that stops at the first failure has already run every other
test; it also passes when run alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from eggsync import _lib, data, egg_grid

pytestmark = pytest.mark.gpu


def grid_noalloc(L, X, eps):
    X = np.ascontiguousarray(X, np.float32)
    n, d = X.shape
    order = np.empty(n, np.int32)
    cell_of = np.empty(n, np.int32)
    start = np.empty(n + 1, np.int32)
    M = C.c_int32(0)
    st = L.egg_sync_grid_noalloc(C.c_void_p(X.ctypes.data), n, d, float(eps), C.c_void_p(order.ctypes.data),
                                 C.c_void_p(cell_of.ctypes.data), C.c_void_p(start.ctypes.data), C.byref(M), None)
    return st, order, cell_of, start[: M.value + 1].copy()


def test_noalloc_grid_equals_grid_twice_in_a_row(eggsync_lib):
    L = eggsync_lib
    inputs = [(data.c1(0)["X"], 0.05), (data.c1(1)["X"][:7000, :], 0.03)]
    for X, eps in inputs:  # two calls in a row share the static scratch
        st, order, cell_of, start = grid_noalloc(L, X, eps)
        assert st == _lib.EGG_OK, L.egg_last_error()
        r_order, r_cell_of, r_start = egg_grid(X, eps)
        assert np.array_equal(order, r_order)
        assert np.array_equal(cell_of, r_cell_of)
        assert np.array_equal(start, r_start)


def test_noalloc_rejects_inputs_beyond_its_limit(eggsync_lib):
    L = eggsync_lib
    X = np.random.default_rng(0).random((65537, 2)).astype(np.float32)
    st, *_ = grid_noalloc(L, X, 0.05)
    assert st == _lib.EGG_ERR_ARG
    assert b"65536" in L.egg_last_error()
    st, *_ = grid_noalloc(L, np.zeros((10, 5), np.float32), 0.05)
    assert st == _lib.EGG_ERR_ARG


def test_noalloc_at_its_limit_with_device_input(eggsync_lib, gpu):
    """n = 65,536 and d = 4, the largest layout the 8 MiB array holds, with
    the points already in device memory (no staging copy); twice in a row,
    and once more after egg_release(), which makes the call look the
    array's address up again."""
    import torch

    L = eggsync_lib
    rng = np.random.default_rng(11)
    centres = rng.uniform(0.1, 0.9, (12, 4))
    X = (centres[rng.integers(0, 12, 65536)] + rng.normal(0, 0.02, (65536, 4))).astype(np.float32)
    X = data.min_max_normalize(X)
    for eps, release in ((0.08, False), (0.05, False), (0.05, True)):
        if release:
            assert L.egg_release() == _lib.EGG_OK
        Xd = torch.from_numpy(X).to(gpu)
        order = torch.empty(65536, dtype=torch.int32, device=gpu)
        cell_of = torch.empty(65536, dtype=torch.int32, device=gpu)
        start = torch.empty(65537, dtype=torch.int32, device=gpu)
        M = C.c_int32(0)
        torch.cuda.synchronize()
        st = L.egg_sync_grid_noalloc(C.c_void_p(Xd.data_ptr()), 65536, 4, eps, C.c_void_p(order.data_ptr()),
                                     C.c_void_p(cell_of.data_ptr()), C.c_void_p(start.data_ptr()), C.byref(M), None)
        assert st == _lib.EGG_OK, L.egg_last_error()
        r_order, r_cell_of, r_start = egg_grid(X, eps)
        assert np.array_equal(order.cpu().numpy(), r_order)
        assert np.array_equal(cell_of.cpu().numpy(), r_cell_of)
        assert np.array_equal(start.cpu().numpy()[: M.value + 1], r_start)


def test_noalloc_rejects_non_finite_input(eggsync_lib):
    L = eggsync_lib
    X = np.random.default_rng(3).random((500, 3)).astype(np.float32)
    X[17, 2] = np.inf
    st, *_ = grid_noalloc(L, X, 0.05)
    assert st == _lib.EGG_ERR_INPUT
    # the next call on finite input works
    X[17, 2] = 0.5
    st, order, cell_of, start = grid_noalloc(L, X, 0.05)
    assert st == _lib.EGG_OK
    r_order, _, r_start = egg_grid(X, 0.05)
    assert np.array_equal(order, r_order) and np.array_equal(start, r_start)
