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
