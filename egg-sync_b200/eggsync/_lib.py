"""ctypes binding of libeggsync.so (the C ABI declared in include/eggsync.h).

There is no fallback: if the shared library is missing or fails to load,
importing this module raises, so no caller can silently run anything but the
CUDA path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(os.environ.get("EGGSYNC_LIB", Path(__file__).resolve().parent.parent / "lib" / "libeggsync.so"))

EGG_OK = 0
EGG_MAX_ITER = 1
EGG_ERR_ARG = -1
EGG_ERR_GEOMETRY = -2
EGG_ERR_INPUT = -3
EGG_ERR_CUDA = -4
EGG_ERR_NO_DEVICE = -5
EGG_ERR_INTERNAL = -6

# every symbol include/eggsync.h declares
EXPORTS = ("egg_opts_default", "egg_sync_run", "egg_sync_step", "egg_sync_grid", "egg_sync_grid_noalloc",
           "egg_sync_batch", "egg_status_str", "egg_last_error", "egg_release", "egg_abi_version",
           "egg_update_counters", "egg_mlp_feature_dim", "egg_mlp_features", "egg_mlp_forward", "egg_mlp_grad",
           "egg_mlp_train", "egg_minmax_normalize", "egg_simple_sync_run", "egg_knn_mean", "egg_mdl_cost",
           "egg_mdl_search", "egg_inject_alloc_failures")

# egg_update_counters slots
UPDATE_COUNTERS = ("points", "cells", "small_pass", "full", "tight_in", "tight_out", "groups_in", "groups_out",
                   "pairs", "pairs_in", "lane_warps", "half_count", "neighbors", "cycles_shared", "cycles_lane",
                   "warp_visits", "cycles_visits", "walk_steps")


class EggMlp(C.Structure):
    _fields_ = [("d", C.c_int32), ("d_in", C.c_int32), ("hidden", C.c_int32), ("k_steps", C.c_int32),
                ("min_count", C.c_int32), ("reserved0", C.c_int32), ("w1", C.c_void_p), ("b1", C.c_void_p), ("w2", C.c_void_p), ("b2", C.c_void_p),
                ("w3", C.c_void_p), ("b3", C.c_void_p)]


class EggMlpTrainOpts(C.Structure):
    _fields_ = [("epochs", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float), ("reserved0", C.c_int32),
                ("seed", C.c_int64)]


class EggOpts(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("loop", C.c_int32), ("stop_rule", C.c_int32),
                ("order_param", C.c_int32), ("profile", C.c_int32), ("full_update", C.c_int32),
                ("positions_out", C.c_void_p), ("labels_mode", C.c_int32), ("batch_tune", C.c_int32),
                ("warm_start", C.c_void_p), ("warm_verify", C.c_int32), ("reserved", C.c_int32 * 3)]


class EggStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("n_cells", C.c_int32),
                ("n_clusters", C.c_int32), ("extra_checks", C.c_int32), ("status_bits", C.c_int32),
                ("workspace_bytes", C.c_int64), ("order_param", C.c_double), ("stage_ms", C.c_float * 6),
                ("total_ms", C.c_float), ("itr_ms", C.POINTER(C.c_float)), ("itr_cap", C.c_int32),
                ("kernel_ms", C.c_float * 4), ("kernel_launches", C.c_int32 * 4), ("launches", C.c_int32),
                ("order_param_lo", C.c_double), ("order_param_hi", C.c_double),
                ("itr_order_param", C.POINTER(C.c_double)), ("warm_started", C.c_int32),
                ("warm_fallback", C.c_int32), ("warm_ms", C.c_float), ("warm_same", C.c_int32),
                ("grid_builds", C.c_int32), ("points_updated", C.c_int64)]


class EggBatchItem(C.Structure):
    _fields_ = [("x", C.c_void_p), ("n", C.c_int64), ("d", C.c_int32), ("eps", C.c_float),
                ("labels", C.c_void_p), ("iterations", C.c_int32), ("converged", C.c_int32),
                ("n_clusters", C.c_int32), ("status", C.c_int32)]


class EggBatchStats(C.Structure):
    _fields_ = [("loop_iterations", C.c_int32), ("groups", C.c_int32), ("launches", C.c_int32),
                ("tuned", C.c_int32), ("update_threads", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("order", C.c_int32), ("reserved0", C.c_int32), ("workspace_bytes", C.c_int64),
                ("total_ms", C.c_float), ("loop_ms", C.c_float), ("tune_ms", C.c_float),
                ("itr_cap", C.c_int32), ("itr_ms", C.POINTER(C.c_float)), ("reserved", C.c_int32 * 2)]


class EggMdlStats(C.Structure):
    _fields_ = [("eps0", C.c_double), ("eps1", C.c_double), ("eps_step", C.c_float), ("eps_best", C.c_float),
                ("candidates", C.c_int32), ("best", C.c_int32), ("n_clusters", C.c_int32),
                ("end_reason", C.c_int32), ("cost_best", C.c_double), ("total_ms", C.c_float),
                ("cap", C.c_int32), ("costs", C.POINTER(C.c_double)), ("eps", C.POINTER(C.c_float)),
                ("clusters", C.POINTER(C.c_int32))]


class EggError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (_status_name(status), msg))
        self.status = status


_lib = None


def _status_name(s):
    try:
        return load().egg_status_str(int(s)).decode()
    except Exception:
        return str(s)


def load():
    """Load libeggsync.so once and declare the prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError("libeggsync.so not found at %s: build it with "
                          "`python -c 'import __graft_entry__ as g; g.build()'`" % LIB_PATH)
    L = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    L.egg_opts_default.argtypes = [C.POINTER(EggOpts)]
    L.egg_opts_default.restype = None
    L.egg_sync_run.argtypes = [vp, C.c_int64, C.c_int32, C.c_float, C.c_float, C.POINTER(EggOpts), vp,
                               C.POINTER(EggStats), vp]
    L.egg_sync_run.restype = C.c_int
    L.egg_sync_step.argtypes = [vp, C.c_int64, C.c_int32, C.c_float, vp, vp, vp, vp]
    L.egg_sync_step.restype = C.c_int
    L.egg_sync_grid.argtypes = [vp, C.c_int64, C.c_int32, C.c_float, vp, vp, vp, C.POINTER(C.c_int32), vp]
    L.egg_sync_grid.restype = C.c_int
    L.egg_sync_grid_noalloc.argtypes = [vp, C.c_int64, C.c_int32, C.c_float, vp, vp, vp, C.POINTER(C.c_int32), vp]
    L.egg_sync_grid_noalloc.restype = C.c_int
    L.egg_sync_batch.argtypes = [C.POINTER(EggBatchItem), C.c_int32, C.POINTER(EggOpts), C.POINTER(EggBatchStats), vp]
    L.egg_sync_batch.restype = C.c_int
    L.egg_status_str.argtypes = [C.c_int]
    L.egg_status_str.restype = C.c_char_p
    L.egg_last_error.argtypes = []
    L.egg_last_error.restype = C.c_char_p
    L.egg_release.argtypes = []
    L.egg_release.restype = C.c_int
    if hasattr(L, "egg_inject_alloc_failures"):  # testing aid (tests/test_capi.py checks every export)
        L.egg_inject_alloc_failures.argtypes = [C.c_int32]
        L.egg_inject_alloc_failures.restype = C.c_int
    L.egg_abi_version.argtypes = []
    L.egg_abi_version.restype = C.c_int
    L.egg_update_counters.argtypes = [C.POINTER(C.c_int64), C.c_int32]
    L.egg_update_counters.restype = C.c_int
    L.egg_simple_sync_run.argtypes = [vp, C.c_int64, C.c_int32, C.c_float, C.c_float, C.c_int32, vp, vp,
                                      C.POINTER(EggStats), vp]
    L.egg_simple_sync_run.restype = C.c_int
    # the eps search (ABI 5); an older library without it still loads, and
    # calling the missing entry point raises AttributeError
    if hasattr(L, "egg_mdl_search"):
        L.egg_knn_mean.argtypes = [vp, C.c_int64, C.c_int32, C.c_int32, C.POINTER(C.c_double), vp]
        L.egg_knn_mean.restype = C.c_int
        L.egg_mdl_cost.argtypes = [vp, C.c_int64, C.c_int32, vp, C.POINTER(C.c_double), C.POINTER(C.c_int32), vp]
        L.egg_mdl_cost.restype = C.c_int
        L.egg_mdl_search.argtypes = [vp, C.c_int64, C.c_int32, C.c_int32, C.c_int32, vp, C.POINTER(EggMdlStats), vp]
        L.egg_mdl_search.restype = C.c_int
    L.egg_minmax_normalize.argtypes = [vp, C.c_int64, C.c_int32, vp, vp, vp, vp]
    L.egg_minmax_normalize.restype = C.c_int
    L.egg_mlp_feature_dim.argtypes = [C.c_int32]
    L.egg_mlp_feature_dim.restype = C.c_int
    L.egg_mlp_features.argtypes = [vp, C.c_int64, C.c_int32, C.c_float, vp]
    L.egg_mlp_features.restype = C.c_int
    L.egg_mlp_forward.argtypes = [C.POINTER(EggMlp), vp, C.c_int64, vp]
    L.egg_mlp_forward.restype = C.c_int
    L.egg_mlp_grad.argtypes = [C.POINTER(EggMlp), vp, vp, C.c_int64, C.POINTER(EggMlp), C.POINTER(C.c_double)]
    L.egg_mlp_grad.restype = C.c_int
    L.egg_mlp_train.argtypes = [C.POINTER(EggMlp), vp, vp, C.c_int64, C.POINTER(EggMlpTrainOpts),
                                C.POINTER(C.c_double)]
    L.egg_mlp_train.restype = C.c_int
    _lib = L
    return L


def check(status):
    """Raise EggError for negative statuses; return the status otherwise."""
    if status < 0:
        msg = load().egg_last_error().decode(errors="replace")
        raise EggError(status, msg)
    return status
