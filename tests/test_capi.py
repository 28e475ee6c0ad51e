"""CPU tests of the C ABI: the library loads, exports every declared entry
point, its struct layouts match the header, and argument errors come back
as status codes (these paths return before any CUDA call)."""
import ctypes as C
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO
from eggsync import _lib

HEADER = REPO / "include" / "eggsync.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(egg_[a-z_]+)\s*\(", text)))


def test_exports_every_declared_symbol(eggsync_lib):
    names = declared_functions()
    assert set(names) == set(_lib.EXPORTS)
    for n in names:
        assert hasattr(eggsync_lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (egg_\w+)", out))
    assert set(names) <= exported
    # nothing but the declared C ABI is exported under the egg_ prefix
    assert exported == set(names)


def test_abi_version_and_status_names(eggsync_lib):
    assert eggsync_lib.egg_abi_version() == 5
    # the normal build collects no interaction counters
    buf = (C.c_int64 * 16)()
    assert eggsync_lib.egg_update_counters(buf, 16) == 0
    assert eggsync_lib.egg_status_str(0) == b"EGG_OK"
    assert eggsync_lib.egg_status_str(-4) == b"EGG_ERR_CUDA"
    assert eggsync_lib.egg_status_str(12345) == b"EGG_UNKNOWN_STATUS"


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "sz.c"
    fields = [("egg_opts", _lib.EggOpts, ["positions_out", "labels_mode", "batch_tune", "warm_start",
                                           "warm_verify"]),
              ("egg_stats", _lib.EggStats, ["stage_ms", "itr_ms", "itr_cap", "itr_order_param", "warm_ms",
                                            "warm_same", "grid_builds", "points_updated"]),
              ("egg_mlp", _lib.EggMlp, ["min_count", "w1", "b3"]),
              ("egg_mlp_train_opts", _lib.EggMlpTrainOpts, ["lr", "seed"]),
              ("egg_batch_item", _lib.EggBatchItem, ["n", "eps", "labels", "status"]),
              ("egg_batch_stats", _lib.EggBatchStats, ["workspace_bytes", "total_ms", "tune_ms", "itr_ms"]),
              ("egg_mdl_stats", _lib.EggMdlStats, ["eps_step", "candidates", "end_reason", "cost_best", "cap",
                                                  "costs", "clusters"])]
    body = "".join('printf("%%zu\\n", sizeof(%s));' % t + "".join(
        'printf("%%zu\\n", offsetof(%s, %s));' % (t, f) for f in fs) for t, _, fs in fields)
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "eggsync.h"\nint main(){%s}\n' % body)
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(REPO / "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    want = []
    for _, S, fs in fields:
        want.append(C.sizeof(S))
        want.extend(getattr(S, f).offset for f in fs)
    assert vals == want
    assert C.sizeof(_lib.EggOpts) == 64


def _run(L, x, n, d, eps, labels):
    return L.egg_sync_run(x, n, d, eps, 0.999, None, labels, None, None)


def test_argument_errors(eggsync_lib):
    L = eggsync_lib
    x = np.zeros((10, 2), np.float32)
    lab = np.zeros(10, np.int32)
    xp, lp = C.c_void_p(x.ctypes.data), C.c_void_p(lab.ctypes.data)
    assert _run(L, None, 10, 2, 0.05, lp) == _lib.EGG_ERR_ARG
    assert _run(L, xp, 10, 2, 0.05, None) == _lib.EGG_ERR_ARG
    assert _run(L, xp, 0, 2, 0.05, lp) == _lib.EGG_ERR_ARG
    assert _run(L, xp, 10, 0, 0.05, lp) == _lib.EGG_ERR_ARG
    assert _run(L, xp, 10, 65, 0.05, lp) == _lib.EGG_ERR_ARG
    assert _run(L, xp, 10, 2, 0.0, lp) == _lib.EGG_ERR_ARG
    assert _run(L, xp, 10, 2, -1.0, lp) == _lib.EGG_ERR_ARG
    assert _run(L, xp, 10, 2, float("nan"), lp) == _lib.EGG_ERR_ARG
    assert b"eps" in L.egg_last_error()
    # eps so large that a dimension has fewer than two cells
    assert _run(L, xp, 10, 2, 5.0, lp) == _lib.EGG_ERR_GEOMETRY
    # eps so small that a dimension has more than 65535 cells
    assert _run(L, xp, 10, 2, 1e-6, lp) == _lib.EGG_ERR_GEOMETRY
    flags = np.zeros(2, np.int32)
    assert L.egg_sync_step(None, 10, 2, 0.05, xp, None, C.c_void_p(flags.ctypes.data), None) == _lib.EGG_ERR_ARG


def test_batch_argument_errors(eggsync_lib):
    L = eggsync_lib
    x = np.zeros((10, 2), np.float32)
    lab = np.zeros(10, np.int32)
    items = (_lib.EggBatchItem * 2)()
    for it in items:
        it.x, it.n, it.d, it.eps, it.labels = x.ctypes.data, 10, 2, 0.05, lab.ctypes.data
    assert L.egg_sync_batch(None, 2, None, None, None) == _lib.EGG_ERR_ARG
    assert L.egg_sync_batch(items, 0, None, None, None) == _lib.EGG_ERR_ARG
    assert L.egg_sync_batch(items, 1025, None, None, None) == _lib.EGG_ERR_ARG
    items[1].eps = 5.0
    assert L.egg_sync_batch(items, 2, None, None, None) == _lib.EGG_ERR_GEOMETRY
    assert L.egg_last_error().startswith(b"item 1:")
    items[1].eps = 0.05
    items[0].labels = None
    assert L.egg_sync_batch(items, 2, None, None, None) == _lib.EGG_ERR_ARG
    items[0].labels = lab.ctypes.data
    opts = _lib.EggOpts()
    opts.stop_rule = 1
    assert L.egg_sync_batch(items, 2, C.byref(opts), None, None) == _lib.EGG_ERR_ARG


def test_simple_sync_argument_errors(eggsync_lib):
    L = eggsync_lib
    x = np.zeros((10, 2), np.float32)
    lab = np.zeros(10, np.int32)
    xp, lp = C.c_void_p(x.ctypes.data), C.c_void_p(lab.ctypes.data)
    assert L.egg_simple_sync_run(None, 10, 2, 0.05, 0.999, 0, lp, None, None, None) == _lib.EGG_ERR_ARG
    assert L.egg_simple_sync_run(xp, 10, 2, 0.05, 0.999, 0, None, None, None, None) == _lib.EGG_ERR_ARG
    assert L.egg_simple_sync_run(xp, 0, 2, 0.05, 0.999, 0, lp, None, None, None) == _lib.EGG_ERR_ARG
    assert L.egg_simple_sync_run(xp, 10, 2, -1.0, 0.999, 0, lp, None, None, None) == _lib.EGG_ERR_ARG
    assert L.egg_simple_sync_run(xp, 10, 2, 0.05, 0.999, -1, lp, None, None, None) == _lib.EGG_ERR_ARG


def test_normalize_argument_errors(eggsync_lib):
    L = eggsync_lib
    x = np.zeros((10, 2), np.float32)
    xp = C.c_void_p(x.ctypes.data)
    assert L.egg_minmax_normalize(None, 10, 2, xp, None, None, None) == _lib.EGG_ERR_ARG
    assert L.egg_minmax_normalize(xp, 0, 2, xp, None, None, None) == _lib.EGG_ERR_ARG
    assert L.egg_minmax_normalize(xp, 10, 65, xp, None, None, None) == _lib.EGG_ERR_ARG


def test_mdl_argument_errors(eggsync_lib):
    L = eggsync_lib
    x = np.zeros((10, 2), np.float32)
    lab = np.zeros(10, np.int32)
    xp, lp = C.c_void_p(x.ctypes.data), C.c_void_p(lab.ctypes.data)
    out = (C.c_double * 2)()
    cost = C.c_double()
    assert L.egg_knn_mean(None, 10, 2, 3, out, None) == _lib.EGG_ERR_ARG
    assert L.egg_knn_mean(xp, 10, 2, 0, out, None) == _lib.EGG_ERR_ARG      # k < 1
    assert L.egg_knn_mean(xp, 10, 2, 32, out, None) == _lib.EGG_ERR_ARG     # k > 31
    assert L.egg_knn_mean(xp, 4, 2, 3, out, None) == _lib.EGG_ERR_ARG       # n < k + 2
    assert L.egg_knn_mean(xp, 10, 65, 3, out, None) == _lib.EGG_ERR_ARG
    assert L.egg_mdl_cost(xp, 10, 2, None, C.byref(cost), None, None) == _lib.EGG_ERR_ARG
    assert L.egg_mdl_cost(xp, 1, 2, lp, C.byref(cost), None, None) == _lib.EGG_ERR_ARG
    assert L.egg_mdl_search(xp, 10, 2, 0, 0, lp, None, None) == _lib.EGG_ERR_ARG
    assert L.egg_mdl_search(xp, 10, 2, 3, -1, lp, None, None) == _lib.EGG_ERR_ARG
    assert L.egg_mdl_search(xp, 10, 2, 3, 0, None, None, None) == _lib.EGG_ERR_ARG


def test_python_front_end_rejects_bad_input(eggsync_lib):
    from eggsync import egg_sync

    with pytest.raises(TypeError):
        egg_sync(np.zeros((10, 2), np.float64), 0.05)
    with pytest.raises(ValueError):
        egg_sync(np.zeros(10, np.float32), 0.05)
    with pytest.raises(_lib.EggError) as e:
        egg_sync(np.zeros((10, 2), np.float32), 5.0)
    assert e.value.status == _lib.EGG_ERR_GEOMETRY


def test_alloc_failure_injection_arguments(eggsync_lib):
    """The error-path testing aid rejects a negative count and clears with 0
    (no device needed)."""
    from eggsync import _lib

    assert eggsync_lib.egg_inject_alloc_failures(-1) == _lib.EGG_ERR_ARG
    assert eggsync_lib.egg_inject_alloc_failures(0) == _lib.EGG_OK
