"""Python access to the oracle (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only to check or to time the reference.  The
product (``egg-sync_b200``) never imports it.

* ``Oracle``: the C restatement in ``egg_oracle.c`` (FP64 update, reference
  decisions), see that file's header for the reference lines it follows.
* ``RefSync``: the reference's own CPU SynC built from its sources
  (``oracle/_ref/libref_sync.so``).
* ``run_ref_egg``: the reference's own EGG-SynC (``oracle/_ref/libref_egg.so``),
  run in a child process with a timeout because it calls ``exit()`` on CUDA
  errors and has no iteration cap.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import build as _build  # noqa: E402

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class Geom(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("d", C.c_int), ("eps", C.c_float), ("side", C.c_float), ("width", C.c_int),
        ("od", C.c_int), ("n_outer", C.c_int64), ("r", C.c_int), ("eps_extra", C.c_float),
        ("r_extra", C.c_int), ("r_half", C.c_int), ("t_eps", C.c_float), ("t_half", C.c_float),
        ("t_extra", C.c_float),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _as_x(X):
    X = np.ascontiguousarray(X, dtype=np.float32)
    if X.ndim != 2:
        raise ValueError("X must be n x d")
    return X


class Oracle:
    """ctypes view of ``libeggoracle.so``."""

    def __init__(self):
        path = _build.build_oracle()
        L = C.CDLL(str(path))
        L.egg_oracle_geometry.argtypes = [C.c_int, C.c_int, C.c_float, C.POINTER(Geom)]
        L.egg_oracle_sq_threshold.argtypes = [C.c_float]
        L.egg_oracle_sq_threshold.restype = C.c_float
        L.egg_oracle_step.argtypes = [_f32p, C.c_int, C.c_int, C.c_float, _f32p, C.c_void_p, C.c_void_p]
        L.egg_oracle_extra_check.argtypes = [_f32p, C.c_int, C.c_int, C.c_float, C.POINTER(C.c_int64)]
        L.egg_oracle_labels.argtypes = [_f32p, C.c_int, C.c_int, C.c_float, _i32p]
        L.egg_oracle_grid.argtypes = [_f32p, C.c_int, C.c_int, C.c_float, _i32p, _i32p, _i32p, C.POINTER(C.c_int)]
        L.egg_oracle_run.argtypes = [_f32p, C.c_int, C.c_int, C.c_float, C.c_int, _i32p, _f32p, _i32p]
        L.egg_oracle_update_sample.argtypes = [_f32p, C.c_int, C.c_int, C.c_float, _i32p, C.c_int, _f32p, _i32p]
        L.egg_oracle_order_parameter.argtypes = [_f32p, C.c_int, C.c_int, C.c_float]
        L.egg_oracle_order_parameter.restype = C.c_double
        L.egg_oracle_order_parameter_egg.argtypes = [_f32p, C.c_int, C.c_int, C.c_float]
        L.egg_oracle_order_parameter_egg.restype = C.c_double
        L.egg_oracle_threads.restype = C.c_int
        L.egg_oracle_step_sample.argtypes = [_f32p, C.c_int, C.c_int, C.c_float, _i32p, C.c_int, _f32p, _i32p,
                                             _i32p]
        L.egg_oracle_ref_annulus_pairs.argtypes = [_f32p, C.c_int, C.c_int, C.c_float, C.POINTER(C.c_int64)]
        L.egg_oracle_ref_annulus_pairs.restype = C.c_int64
        L.egg_oracle_set_box_mode.argtypes = [C.c_int]
        L.egg_oracle_set_box_mode.restype = None
        L.egg_oracle_set_face_fma.argtypes = [C.c_int]
        L.egg_oracle_set_face_fma.restype = None
        self.L = L

    def set_face_fma(self, on: bool):
        """Rounding of the box-distance face offsets (see egg_oracle.c)."""
        self.L.egg_oracle_set_face_fma(1 if on else 0)

    def set_box_mode(self, exact: bool):
        """False (default): the reference's cell test; True: the true minimum box distance."""
        self.L.egg_oracle_set_box_mode(1 if exact else 0)

    def threads(self):
        return self.L.egg_oracle_threads()

    def geometry(self, n, d, eps):
        g = Geom()
        if self.L.egg_oracle_geometry(int(n), int(d), float(eps), C.byref(g)) != 0:
            raise ValueError("degenerate geometry (cell width < 2)")
        return g

    def sq_threshold(self, e):
        return self.L.egg_oracle_sq_threshold(float(e))

    def step(self, X, eps, want_delta=False):
        """One iteration: (X_next, counts, flag[, delta64])."""
        X = _as_x(X)
        n, d = X.shape
        out = np.empty_like(X)
        counts = np.empty(n, np.int32)
        delta = np.empty((n, d), np.float64) if want_delta else None
        flag = self.L.egg_oracle_step(X, n, d, float(eps), out, counts.ctypes.data,
                                      delta.ctypes.data if want_delta else None)
        if flag < 0:
            raise ValueError("oracle step failed")
        return (out, counts, flag, delta) if want_delta else (out, counts, flag)

    def step_sample(self, X, eps, idx):
        """One iteration for the sampled points only: (X_next rows, counts, violations)."""
        X = _as_x(X)
        idx = np.ascontiguousarray(idx, np.int32)
        out = np.empty((len(idx), X.shape[1]), np.float32)
        cnt = np.empty(len(idx), np.int32)
        viol = np.empty(len(idx), np.int32)
        if self.L.egg_oracle_step_sample(X, X.shape[0], X.shape[1], float(eps), idx, len(idx), out, cnt, viol) < 0:
            raise ValueError("oracle step failed")
        return out, cnt, viol

    def extra_check(self, X, eps):
        X = _as_x(X)
        pairs = C.c_int64(0)
        ok = self.L.egg_oracle_extra_check(X, X.shape[0], X.shape[1], float(eps), C.byref(pairs))
        return ok, pairs.value

    def ref_annulus_pairs(self, X, eps):
        """(total, largest per point) of the pairs the reference's extra check
        lists on X (EGG_SynC.cu:767-878)."""
        X = _as_x(X)
        worst = C.c_int64(0)
        total = self.L.egg_oracle_ref_annulus_pairs(X, X.shape[0], X.shape[1], float(eps), C.byref(worst))
        return int(total), int(worst.value)

    def labels(self, X, eps):
        X = _as_x(X)
        lab = np.empty(X.shape[0], np.int32)
        self.L.egg_oracle_labels(X, X.shape[0], X.shape[1], float(eps), lab)
        return lab

    def grid(self, X, eps):
        X = _as_x(X)
        n = X.shape[0]
        order = np.empty(n, np.int32)
        cell_of = np.empty(n, np.int32)
        start = np.empty(n + 1, np.int32)
        M = C.c_int(0)
        self.L.egg_oracle_grid(X, n, X.shape[1], float(eps), order, cell_of, start, C.byref(M))
        return order, cell_of, start[: M.value + 1].copy()

    def run(self, X, eps, max_iter=0):
        """Full loop: (labels, iterations, final X, per-iteration flags)."""
        X = _as_x(X)
        n, d = X.shape
        lab = np.empty(n, np.int32)
        fin = np.empty_like(X)
        cap = max_iter if max_iter > 0 else 100000
        flags = np.zeros(cap, np.int32)
        it = self.L.egg_oracle_run(X, n, d, float(eps), int(max_iter), lab, fin, flags)
        if it < 0:
            raise ValueError("oracle run failed")
        return lab, it, fin, flags[:it].copy()

    def update_sample(self, X, eps, idx):
        X = _as_x(X)
        idx = np.ascontiguousarray(idx, np.int32)
        out = np.empty((len(idx), X.shape[1]), np.float32)
        cnt = np.empty(len(idx), np.int32)
        self.L.egg_oracle_update_sample(X, X.shape[0], X.shape[1], float(eps), idx, len(idx), out, cnt)
        return out, cnt

    def order_parameter(self, X, eps):
        """Brute-force neighbourhoods (the reference CPU SynC's)."""
        X = _as_x(X)
        return self.L.egg_oracle_order_parameter(X, X.shape[0], X.shape[1], float(eps))

    def order_parameter_egg(self, X, eps):
        """Neighbourhoods of the EGG-SynC update (exact FP64)."""
        X = _as_x(X)
        return self.L.egg_oracle_order_parameter_egg(X, X.shape[0], X.shape[1], float(eps))


class RefSync:
    """The reference's own CPU SynC (``SynC.cpp``), compiled from its sources."""

    def __init__(self, path=None):
        path = Path(path) if path else _build.REF_DIR / "libref_sync.so"
        if not path.exists():
            if _build.ref_available():
                _build.build_ref(with_gpu=False)
            else:
                raise FileNotFoundError(str(path))
        import torch  # noqa: F401  (loads libc10/libtorch_cpu for the reference's ATen use)

        L = C.CDLL(str(path))
        L.ref_sync_run.argtypes = [_f32p, C.c_int, C.c_int, C.c_float, C.c_float, _i32p, C.POINTER(C.c_int)]
        L.ref_sync_serial_run.argtypes = L.ref_sync_run.argtypes
        L.ref_sync_step_sample.argtypes = [_f32p, C.c_int, C.c_int, C.c_float, _i32p, C.c_int, _f32p, _i32p, _f32p]
        L.ref_sync_threads.restype = C.c_int
        self.L = L

    def threads(self):
        return self.L.ref_sync_threads()

    def run(self, X, eps, lam=1 - 1e-3, parallel=True):
        X = _as_x(X)
        lab = np.empty(X.shape[0], np.int32)
        it = C.c_int(0)
        fn = self.L.ref_sync_run if parallel else self.L.ref_sync_serial_run
        fn(X, X.shape[0], X.shape[1], float(eps), float(lam), lab, C.byref(it))
        return lab, it.value

    def step_sample(self, X, eps, idx):
        X = _as_x(X)
        idx = np.ascontiguousarray(idx, np.int32)
        out = np.empty((len(idx), X.shape[1]), np.float32)
        cnt = np.empty(len(idx), np.int32)
        r = np.empty(len(idx), np.float32)
        self.L.ref_sync_step_sample(X, X.shape[0], X.shape[1], float(eps), idx, len(idx), out, cnt, r)
        return out, cnt, r


_REF_EGG_CHILD = r"""
import sys, json, time, ctypes as C, numpy as np, torch
X = np.load(sys.argv[2]).astype(np.float32)
if torch.cuda.is_available():
    torch.zeros(1, device="cuda")  # the CUDA context exists before the timed call
eps = float(sys.argv[3])
L = C.CDLL(sys.argv[1])
n, d = X.shape
lab = np.empty(n, np.int32)
it = C.c_int(0)
st = np.zeros(6, np.float32)
f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
L.ref_egg_run.argtypes = [f32p, C.c_int, C.c_int, C.c_float, i32p, C.POINTER(C.c_int), f32p]
Xc = np.ascontiguousarray(X)
t0 = time.perf_counter()
rc = L.ref_egg_run(Xc, n, d, eps, lab, C.byref(it), st)
wall = time.perf_counter() - t0
np.save(sys.argv[4], lab)
sys.stderr.write("REF_EGG_RESULT " + json.dumps({"rc": rc, "iters": it.value, "stage_times": st.tolist(),
                                                 "wall_s": wall}) + "\n")
"""

# The reference EGG-SynC's extra check counts its pairs with
# atomicInc(counter, n * n) and sizes its pair list with int arithmetic
# (EGG_SynC.cu:878, 1010, 1449-1450): the int product n * n wraps (mod 2^32,
# read as unsigned by atomicInc, which restarts at 0 past that limit), and
# 2 * count must fit in an int.  For n <= 32768 every possible count is
# inside both limits; above it the reference is defined only while the
# counts of the iterations that run the extra check stay below
# ref_egg_pair_limit(n) (counted with Oracle.ref_annulus_pairs first).
REF_EGG_MAX_N = 32768


def ref_egg_pair_limit(n):
    """Largest number of extra-check pairs + 1 the reference handles at n points."""
    wrap = (n * n) % (1 << 32)
    return min(1 << 30, wrap)


def run_ref_egg(X, eps, timeout=600, workdir=None, max_pairs=None, info_out=None):
    """Run the reference EGG-SynC on X in a child process.

    For n > 32768 the caller passes ``max_pairs``, the largest pair count of
    the reference's extra check over the run (counted beforehand); the run
    is refused unless it is below ``ref_egg_pair_limit(n)``.  ``info_out``
    (a dict) receives the child's wall time of the call.

    Returns (labels, iterations, stage_times)."""
    import tempfile

    X = _as_x(X)
    if X.shape[0] > REF_EGG_MAX_N and (max_pairs is None or max_pairs >= ref_egg_pair_limit(X.shape[0])):
        raise ValueError("reference EGG-SynC at n = %d needs a pair count below %d (got %s)" %
                         (X.shape[0], ref_egg_pair_limit(X.shape[0]), max_pairs))
    so = _build.REF_DIR / "libref_egg.so"
    if not so.exists():
        raise FileNotFoundError(str(so))
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        xin = os.path.join(td, "x.npy")
        lout = os.path.join(td, "lab.npy")
        np.save(xin, X)
        r = subprocess.run([sys.executable, "-c", _REF_EGG_CHILD, str(so), xin, repr(float(eps)), lout],
                           capture_output=True, text=True, timeout=timeout)
        info = None
        for line in r.stderr.splitlines():
            if line.startswith("REF_EGG_RESULT "):
                info = json.loads(line[len("REF_EGG_RESULT "):])
        if r.returncode != 0 or info is None or info["rc"] != 0:
            raise RuntimeError("reference EGG-SynC failed (rc=%s): %s" % (r.returncode, r.stderr[-2000:]))
        if info_out is not None:
            info_out.update(info)
        return np.load(lout), info["iters"], info["stage_times"]


_REF_SIMPLE_CHILD = r"""
import sys, json, ctypes as C, numpy as np, torch
X = np.load(sys.argv[2]).astype(np.float32)
eps, lam = float(sys.argv[3]), float(sys.argv[4])
L = C.CDLL(sys.argv[1])
n, d = X.shape
lab = np.empty(n, np.int32)
it = C.c_int(0)
f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
L.ref_simple_run.argtypes = [f32p, C.c_int, C.c_int, C.c_float, C.c_float, i32p, C.POINTER(C.c_int)]
rc = L.ref_simple_run(np.ascontiguousarray(X), n, d, eps, lam, lab, C.byref(it))
np.save(sys.argv[5], lab)
sys.stderr.write("REF_SIMPLE_RESULT " + json.dumps({"rc": rc, "iters": it.value}) + "\n")
"""


def run_ref_simple(X, eps, lam=1 - 1e-3, timeout=600, workdir=None):
    """Run the reference brute-force GPU SynC (simple_GPU_SynC.cu) on X in a
    child process.  Returns (labels, iterations)."""
    import tempfile

    X = _as_x(X)
    so = _build.REF_DIR / "libref_simple.so"
    if not so.exists():
        raise FileNotFoundError(str(so))
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        xin = os.path.join(td, "x.npy")
        lout = os.path.join(td, "lab.npy")
        np.save(xin, X)
        r = subprocess.run([sys.executable, "-c", _REF_SIMPLE_CHILD, str(so), xin, repr(float(eps)),
                            repr(float(lam)), lout], capture_output=True, text=True, timeout=timeout)
        info = None
        for line in r.stderr.splitlines():
            if line.startswith("REF_SIMPLE_RESULT "):
                info = json.loads(line[len("REF_SIMPLE_RESULT "):])
        if r.returncode != 0 or info is None or info["rc"] != 0:
            raise RuntimeError("reference GPU SynC failed (rc=%s): %s" % (r.returncode, r.stderr[-2000:]))
        return np.load(lout), info["iters"]


def ari(a, b):
    """Adjusted Rand index with every -1 (noise) mapped to its own singleton."""
    a = np.asarray(a).astype(np.int64).copy()
    b = np.asarray(b).astype(np.int64).copy()
    n = len(a)
    if n != len(b):
        raise ValueError("length mismatch")
    for v in (a, b):
        neg = v < 0
        v[neg] = v.max(initial=0) + 1 + np.arange(int(neg.sum()))
    _, ai = np.unique(a, return_inverse=True)
    _, bi = np.unique(b, return_inverse=True)
    pairs = ai.astype(np.int64) * (bi.max() + 1) + bi
    _, nij = np.unique(pairs, return_counts=True)
    ai_c = np.bincount(ai)
    bi_c = np.bincount(bi)

    def c2(x):
        x = x.astype(np.float64)
        return (x * (x - 1) / 2).sum()

    sij, sa, sb = c2(nij), c2(ai_c), c2(bi_c)
    tot = n * (n - 1) / 2.0
    exp = sa * sb / tot if tot > 0 else 0.0
    mx = 0.5 * (sa + sb)
    if mx == exp:
        return 1.0
    return float((sij - exp) / (mx - exp))


def same_partition(a, b):
    """True when a and b are identical up to relabelling (noise = singletons)."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return False
    if not np.array_equal(a < 0, b < 0):
        return False
    m = a >= 0
    if not m.any():
        return True
    pairs = np.unique(np.stack([a[m], b[m]], 1), axis=0)
    return len(np.unique(pairs[:, 0])) == len(pairs) and len(np.unique(pairs[:, 1])) == len(pairs)
