"""Python front end of the B200 EGG-SynC (mirrors python/algorithms.py).

The reference's front end JIT-builds a torch extension and exposes
``EGG_SynC(D, eps) -> impl.EGG_SynC_wrapper(D, eps)``
(python/algorithms.py:6-17, 110-111; boundary src/maps/map.cpp:31-33).
Here ``impl`` is a thin object over the C ABI of libeggsync.so with the same
method name, argument meaning and return value:

    C, itr_times, stage_times, space = EGG_SynC(D, eps)

* ``C``: float32 tensor (n,), the compacted final cell index of each point
  whose final cell holds more than one point, else -1 (EGG_SynC.cu:1205-1227,
  1527-1541);
* ``itr_times``: float32 tensor (#iterations,), seconds per iteration;
* ``stage_times``: float32 tensor (6,), seconds in the reference's stage slots
  (allocating, build structure, update, extra check, clustering, copy-out);
* ``space``: int32 tensor (1,), device workspace bytes.

Unlike the reference, ``D`` may live on the host or on a CUDA device, its
dtype must be float32 (checked; the reference only asserts it through
``data_ptr<float>``), and failures raise ``EggError`` instead of exiting.
``lam`` is accepted (the reference's EGG path ignores it, EGG_SynC.cu:1233).
"""
from __future__ import annotations

import ctypes as C
from typing import Tuple

import numpy as np

from . import _lib
from ._lib import EggError, EggOpts, EggStats, check

DEFAULT_LAMBDA = 1 - 1e-3


def _torch():
    import torch

    return torch


def _prepare(X):
    """Return (pointer, n, d, keepalive, device_index or None, stream pointer)."""
    if isinstance(X, np.ndarray):
        if X.dtype != np.float32:
            raise TypeError("EGG-SynC expects float32 data, got %s" % X.dtype)
        A = np.ascontiguousarray(X)
        if A.ndim != 2:
            raise ValueError("D must be a 2-D n x d array")
        return A.ctypes.data, A.shape[0], A.shape[1], A, None, None
    torch = _torch()
    if not isinstance(X, torch.Tensor):
        raise TypeError("D must be a torch.Tensor or numpy.ndarray")
    if X.dtype != torch.float32:
        raise TypeError("EGG-SynC expects a float32 tensor, got %s" % X.dtype)
    if X.dim() != 2:
        raise ValueError("D must be a 2-D n x d tensor")
    T = X.contiguous()
    if T.is_cuda:
        return T.data_ptr(), T.shape[0], T.shape[1], T, T.device.index, torch.cuda.current_stream(T.device).cuda_stream
    return T.data_ptr(), T.shape[0], T.shape[1], T, None, None


class _DeviceGuard:
    def __init__(self, idx):
        self.idx = idx
        self.ctx = None

    def __enter__(self):
        if self.idx is not None:
            self.ctx = _torch().cuda.device(self.idx)
            self.ctx.__enter__()

    def __exit__(self, *a):
        if self.ctx is not None:
            self.ctx.__exit__(*a)


def _out_ptr(buf, n, dtype_np, what):
    if isinstance(buf, np.ndarray):
        if buf.dtype != dtype_np or buf.size != n or not buf.flags.c_contiguous:
            raise ValueError("%s must be a contiguous %s array of %d entries" % (what, np.dtype(dtype_np), n))
        return buf.ctypes.data
    torch = _torch()
    tdt = {np.int32: torch.int32, np.float32: torch.float32}[dtype_np]
    if buf.dtype != tdt or buf.numel() != n or not buf.is_contiguous():
        raise ValueError("%s must be a contiguous %s tensor of %d entries" % (what, tdt, n))
    return buf.data_ptr()


def egg_sync(D, eps: float, lam: float = DEFAULT_LAMBDA, max_iter: int = 0, loop: str = "graph",
             labels_out=None, profile: bool = False, full_update: bool = False,
             positions_out=None, stop_rule: str = "flag", order_param: int = 0,
             labels_mode: str = "union_find", warm_start=None, warm_verify: bool = False) -> Tuple[object, dict]:
    """Run EGG-SynC; return (int32 labels, stats dict).

    ``labels_out`` may be a preallocated int32 numpy array or torch tensor
    (host or device) of n entries; by default a host numpy array is returned.
    ``loop`` is "graph" (device-resident loop) or "host".  ``profile`` times
    every kernel group with CUDA events (host-driven loop).  ``full_update``
    recomputes every point in every iteration (the default reuses results
    whose inputs did not change; both give identical bits).
    ``positions_out`` (optional n x d float32 buffer) receives the final
    positions.  ``stop_rule`` "flag" is the reference EGG-SynC's convergence
    test; "lambda" stops once the certified lower bound of the FP64 local
    order parameter reaches ``lam``.  ``order_param`` 1 reports the order
    parameter of the final positions, 2 that of every iteration.
    ``warm_start`` (an ``eggsync.warm.Model``, d <= 3) displaces the input by
    the network's prediction before the plain loop; ``warm_verify`` also runs
    the plain loop from the input and returns it when the partitions differ."""
    L = _lib.load()
    ptr, n, d, keep, dev, stream = _prepare(D)
    if labels_out is None:
        labels_out = np.empty(n, np.int32)
    lptr = _out_ptr(labels_out, n, np.int32, "labels_out")
    opts = EggOpts()
    L.egg_opts_default(C.byref(opts))
    opts.max_iter = int(max_iter)
    opts.loop = {"graph": 0, "host": 1}[loop]
    opts.profile = 1 if profile else 0
    opts.full_update = 1 if full_update else 0
    opts.stop_rule = {"flag": 0, "lambda": 1}[stop_rule]
    opts.order_param = int(order_param)
    opts.labels_mode = {"union_find": 0, "cells": 1}[labels_mode]
    if positions_out is not None:
        opts.positions_out = _out_ptr(positions_out, n * d, np.float32, "positions_out")
    mlp = None
    if warm_start is not None:
        mlp = warm_start.struct()
        opts.warm_start = C.addressof(mlp)
        opts.warm_verify = 1 if warm_verify else 0
    stats = EggStats()
    cap = opts.max_iter if opts.max_iter > 0 else 1000
    itr = (C.c_float * cap)()
    stats.itr_ms = C.cast(itr, C.POINTER(C.c_float))
    stats.itr_cap = cap
    itr_r = (C.c_double * (2 * cap))()
    stats.itr_order_param = C.cast(itr_r, C.POINTER(C.c_double))
    with _DeviceGuard(dev):
        st = check(L.egg_sync_run(C.c_void_p(ptr), n, d, float(eps), float(lam), C.byref(opts), C.c_void_p(lptr),
                                  C.byref(stats), C.c_void_p(stream) if stream else None))
    del keep
    info = {
        "status": int(st),
        "iterations": int(stats.iterations),
        "converged": bool(stats.converged),
        "n_cells": int(stats.n_cells),
        "n_clusters": int(stats.n_clusters),
        "extra_checks": int(stats.extra_checks),
        "status_bits": int(stats.status_bits),
        "workspace_bytes": int(stats.workspace_bytes),
        "stage_ms": [float(v) for v in stats.stage_ms],
        "total_ms": float(stats.total_ms),
        "itr_ms": [float(itr[i]) for i in range(min(stats.iterations, cap))],
        "kernel_ms": dict(zip(("build", "cell_sums", "update", "extra"), [float(v) for v in stats.kernel_ms])),
        "kernel_launches": dict(zip(("build", "cell_sums", "update", "extra"),
                                    [int(v) for v in stats.kernel_launches])),
        "launches": int(stats.launches),
        "order_param": (float(stats.order_param_lo), float(stats.order_param_hi)),
        "itr_order_param": [(float(itr_r[2 * k]), float(itr_r[2 * k + 1]))
                            for k in range(min(stats.iterations, cap))] if (order_param == 2 or
                                                                             stop_rule == "lambda") else [],
        "warm_started": bool(stats.warm_started),
        "warm_fallback": bool(stats.warm_fallback),
        "warm_same": bool(stats.warm_same),
        "warm_ms": float(stats.warm_ms),
        "grid_builds": int(stats.grid_builds),
        "points_updated": int(stats.points_updated),
    }
    del mlp
    return labels_out, info


def egg_step(D, eps: float):
    """One iteration from D: (x_next float32 n x d, counts int32 n, flags (update, after extra check))."""
    L = _lib.load()
    ptr, n, d, keep, dev, stream = _prepare(D)
    out = np.empty((n, d), np.float32)
    cnt = np.empty(n, np.int32)
    flags = np.zeros(2, np.int32)
    with _DeviceGuard(dev):
        check(L.egg_sync_step(C.c_void_p(ptr), n, d, float(eps), C.c_void_p(out.ctypes.data),
                              C.c_void_p(cnt.ctypes.data), C.c_void_p(flags.ctypes.data),
                              C.c_void_p(stream) if stream else None))
    del keep
    return out, cnt, (int(flags[0]), int(flags[1]))


def egg_grid(D, eps: float, out=None):
    """The double grid of D: (order, cell_of, cell_start) as int32 arrays.

    ``out`` (optional): three preallocated int32 buffers (numpy arrays or
    torch tensors, host or device) of n, n and n + 1 entries; they are
    filled and returned, cell_start sliced to the n_cells + 1 used entries."""
    L = _lib.load()
    ptr, n, d, keep, dev, stream = _prepare(D)
    if out is None:
        out = (np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n + 1, np.int32))
    order, cell_of, start = out
    ptrs = [_out_ptr(b, m, np.int32, w) for b, m, w in ((order, n, "order"), (cell_of, n, "cell_of"),
                                                         (start, n + 1, "cell_start"))]
    M = C.c_int32(0)
    with _DeviceGuard(dev):
        check(L.egg_sync_grid(C.c_void_p(ptr), n, d, float(eps), C.c_void_p(ptrs[0]), C.c_void_p(ptrs[1]),
                              C.c_void_p(ptrs[2]), C.byref(M), C.c_void_p(stream) if stream else None))
    del keep
    return order, cell_of, start[: M.value + 1]


def egg_sync_batch(instances, max_iter: int = 0, full_update: bool = False, tune: str = "auto",
                   loop: str = "graph", labels_out=None):
    """Run many instances in one batched call (one CUDA graph for all).

    ``instances``: sequence of (D, eps) pairs; each D is an n x d float32
    numpy array or torch tensor (host or CUDA), sizes and dimensions may
    differ.  ``labels_out`` (optional) gives one preallocated int32 buffer per
    instance.  ``tune``: "auto" (autotune once per workload, cached), "off"
    (default configuration) or "again".  Returns (list of (labels, info),
    batch info).  Every instance's labels and iteration count equal those of
    ``egg_sync`` on it alone."""
    L = _lib.load()
    m = len(instances)
    items = (_lib.EggBatchItem * m)()
    keep = []
    outs = []
    dev = None
    stream = None
    for k, (D, eps) in enumerate(instances):
        ptr, n, d, kp, dv, st = _prepare(D)
        keep.append(kp)
        if dv is not None:
            if dev is not None and dv != dev:
                raise ValueError("all device inputs of a batch must be on one device")
            dev, stream = dv, st
        out = labels_out[k] if labels_out is not None else np.empty(n, np.int32)
        outs.append(out)
        it = items[k]
        it.x, it.n, it.d, it.eps = ptr, n, d, float(eps)
        it.labels = _out_ptr(out, n, np.int32, "labels_out[%d]" % k)
    opts = EggOpts()
    L.egg_opts_default(C.byref(opts))
    opts.max_iter = int(max_iter)
    opts.full_update = 1 if full_update else 0
    opts.batch_tune = {"auto": 0, "off": 1, "again": 2}[tune]
    opts.loop = {"graph": 0, "host": 1}[loop]
    stats = _lib.EggBatchStats()
    cap = opts.max_iter if opts.max_iter > 0 else 1000
    itr = (C.c_float * cap)()
    stats.itr_ms = C.cast(itr, C.POINTER(C.c_float))
    stats.itr_cap = cap
    with _DeviceGuard(dev):
        check(L.egg_sync_batch(items, m, C.byref(opts), C.byref(stats), C.c_void_p(stream) if stream else None))
    del keep
    results = []
    for k in range(m):
        it = items[k]
        if it.status < 0:
            raise EggError(it.status, "instance %d" % k)
        results.append((outs[k], {"iterations": int(it.iterations), "converged": bool(it.converged),
                                  "n_clusters": int(it.n_clusters), "status": int(it.status)}))
    binfo = {f: getattr(stats, f) for f, _ in _lib.EggBatchStats._fields_
             if not f.startswith("reserved") and f not in ("itr_ms", "itr_cap")}
    binfo = {k: (float(v) if isinstance(v, float) else int(v)) for k, v in binfo.items()}
    binfo["itr_ms"] = [float(itr[i]) for i in range(min(stats.loop_iterations, cap))]
    return results, binfo


def simple_sync(D, eps: float, lam: float = DEFAULT_LAMBDA, max_iter: int = 0, labels_out=None,
                positions_out=None):
    """Brute-force GPU SynC (simple_GPU_SynC.cu semantics): (int32 labels, info).
    ``positions_out`` (optional n x d float32) receives the final positions."""
    L = _lib.load()
    ptr, n, d, keep, dev, stream = _prepare(D)
    if labels_out is None:
        labels_out = np.empty(n, np.int32)
    lptr = _out_ptr(labels_out, n, np.int32, "labels_out")
    pptr = _out_ptr(positions_out, n * d, np.float32, "positions_out") if positions_out is not None else None
    stats = EggStats()
    cap = max_iter if max_iter > 0 else 100
    itr = (C.c_float * cap)()
    stats.itr_ms = C.cast(itr, C.POINTER(C.c_float))
    stats.itr_cap = cap
    with _DeviceGuard(dev):
        st = check(L.egg_simple_sync_run(C.c_void_p(ptr), n, d, float(eps), float(lam), int(max_iter),
                                         C.c_void_p(lptr), C.c_void_p(pptr) if pptr else None, C.byref(stats),
                                         C.c_void_p(stream) if stream else None))
    del keep
    return labels_out, {"status": int(st), "iterations": int(stats.iterations), "converged": bool(stats.converged),
                        "n_clusters": int(stats.n_clusters), "r_local": float(stats.order_param),
                        "itr_ms": [float(itr[i]) for i in range(min(stats.iterations, cap))],
                        "stage_ms": [float(v) for v in stats.stage_ms], "total_ms": float(stats.total_ms),
                        "workspace_bytes": int(stats.workspace_bytes)}


def normalize(D, out=None):
    """Per-dimension min-max normalisation on the GPU (python/data.py:100-103
    semantics, float32).  D: n x d float32 numpy array or torch tensor (host
    or CUDA); the result has D's type and device (``out`` may be D itself).
    Returns (normalised points, per-dimension minima, maxima)."""
    L = _lib.load()
    ptr, n, d, keep, dev, stream = _prepare(D)
    if out is None:
        if isinstance(D, np.ndarray):
            out = np.empty((n, d), np.float32)
        else:
            out = _torch().empty((n, d), dtype=_torch().float32, device=D.device)
    optr = _out_ptr(out, n * d, np.float32, "out")
    lo = np.empty(d, np.float32)
    hi = np.empty(d, np.float32)
    with _DeviceGuard(dev):
        check(L.egg_minmax_normalize(C.c_void_p(ptr), n, d, C.c_void_p(optr), C.c_void_p(lo.ctypes.data),
                                     C.c_void_p(hi.ctypes.data), C.c_void_p(stream) if stream else None))
    del keep
    return out, lo, hi


def knn_mean(D, k: int):
    """Mean distance of the points to their k-th and (k+1)-th nearest other
    point (python/SynCTorch.py:112-137, NN(k, D) and NN(k+1, D)), on the
    GPU.  Returns (NN(k), NN(k+1))."""
    L = _lib.load()
    ptr, n, d, keep, dev, stream = _prepare(D)
    out = (C.c_double * 2)()
    with _DeviceGuard(dev):
        check(L.egg_knn_mean(C.c_void_p(ptr), n, d, int(k), out, C.c_void_p(stream) if stream else None))
    del keep
    return float(out[0]), float(out[1])


def mdl_cost(D, labels) -> Tuple[float, int]:
    """Coding cost of the clustering given by ``labels`` (>= 0: cluster id,
    -1: outlier), L_Clust_Outl (python/SynCTorch.py:265-314), on the GPU.
    Returns (cost, number of clusters)."""
    L = _lib.load()
    ptr, n, d, keep, dev, stream = _prepare(D)
    lab = labels
    if isinstance(lab, np.ndarray):
        lab = np.ascontiguousarray(lab, np.int32)
    lptr = _out_ptr(lab, n, np.int32, "labels")
    cost = C.c_double()
    k = C.c_int32()
    with _DeviceGuard(dev):
        check(L.egg_mdl_cost(C.c_void_p(ptr), n, d, C.c_void_p(lptr), C.byref(cost), C.byref(k),
                             C.c_void_p(stream) if stream else None))
    del keep
    return float(cost.value), int(k.value)


def mdl_search(D, k: int, max_candidates: int = 0, labels_out=None):
    """The full-SynC eps search, Sync(D, k) (python/SynCTorch.py:349-372):
    eps from NN(k) in steps of NN(k+1) - NN(k), each eps clustered with
    EGG-SynC and costed by L_Clust_Outl, stopping after the first clustering
    with one cluster; returns (labels of the clustering of least cost, info)."""
    L = _lib.load()
    ptr, n, d, keep, dev, stream = _prepare(D)
    if labels_out is None:
        labels_out = np.empty(n, np.int32)
    lptr = _out_ptr(labels_out, n, np.int32, "labels_out")
    cap = max_candidates if max_candidates > 0 else 256
    costs = (C.c_double * cap)()
    epss = (C.c_float * cap)()
    ks = (C.c_int32 * cap)()
    st = _lib.EggMdlStats()
    st.cap = cap
    st.costs = C.cast(costs, C.POINTER(C.c_double))
    st.eps = C.cast(epss, C.POINTER(C.c_float))
    st.clusters = C.cast(ks, C.POINTER(C.c_int32))
    with _DeviceGuard(dev):
        check(L.egg_mdl_search(C.c_void_p(ptr), n, d, int(k), int(max_candidates), C.c_void_p(lptr), C.byref(st),
                               C.c_void_p(stream) if stream else None))
    del keep
    m = min(st.candidates, cap)
    info = {"eps0": st.eps0, "eps1": st.eps1, "eps_step": st.eps_step, "eps_best": st.eps_best,
            "candidates": st.candidates, "best": st.best, "n_clusters": st.n_clusters,
            "end_reason": {0: "one cluster", 1: "candidate cap", 2: "eps beyond the grid"}[st.end_reason],
            "cost_best": st.cost_best, "total_ms": st.total_ms, "costs": [costs[i] for i in range(m)],
            "eps": [epss[i] for i in range(m)], "clusters": [ks[i] for i in range(m)]}
    return labels_out, info


class _Impl:
    """Stand-in for the reference's JIT module object ``impl``."""

    @staticmethod
    def EGG_SynC_wrapper(D, eps, lam=DEFAULT_LAMBDA):
        torch = _torch()
        lab, info = egg_sync(D, eps, lam)
        C_ = torch.from_numpy(lab.astype(np.float32))
        itr_times = torch.tensor([t / 1000.0 for t in info["itr_ms"]], dtype=torch.float32)
        stage_times = torch.tensor([t / 1000.0 for t in info["stage_ms"]], dtype=torch.float32)
        space = torch.tensor([min(info["workspace_bytes"], 2**31 - 1)], dtype=torch.int32)
        return [C_, itr_times, stage_times, space]


    @staticmethod
    def GPU_DynamicalClustering_wrapper(D, eps, lam=DEFAULT_LAMBDA):
        torch = _torch()
        lab, info = simple_sync(D, eps, lam)
        C_ = torch.from_numpy(lab.astype(np.float32))
        itr_times = torch.tensor([t / 1000.0 for t in info["itr_ms"]], dtype=torch.float32)
        stage_times = torch.tensor([t / 1000.0 for t in info["stage_ms"]], dtype=torch.float32)
        space = torch.tensor([min(info["workspace_bytes"], 2**31 - 1)], dtype=torch.int32)
        return [C_, itr_times, stage_times, space]


impl = _Impl()


def EGG_SynC(D, eps, lam=DEFAULT_LAMBDA):
    """python/algorithms.py:110-111 ``EGG_SynC(D, eps)``, with the optional lambda."""
    return impl.EGG_SynC_wrapper(D, eps, lam)


def GPU_DynamicalClustering(D, eps, lam=DEFAULT_LAMBDA, call=None):
    """python/algorithms.py:33-34: the brute-force GPU SynC."""
    return impl.GPU_DynamicalClustering_wrapper(D, eps, lam)


__all__ = ["EGG_SynC", "GPU_DynamicalClustering", "impl", "egg_sync", "egg_sync_batch", "egg_step", "egg_grid",
           "normalize", "simple_sync", "EggError", "DEFAULT_LAMBDA"]
