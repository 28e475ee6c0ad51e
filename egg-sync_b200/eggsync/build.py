"""Compile libeggsync.so (sm_100a) in-tree.

``build()`` runs nvcc on every ``csrc/*.cu`` in parallel and links them into
``egg-sync_b200/lib/libeggsync.so``.  The shared library is plain C ABI
(``include/eggsync.h``); it links only the CUDA runtime.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent.parent          # egg-sync_b200/
REPO = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
INCLUDE = REPO / "include"
LIB = LIBDIR / "libeggsync.so"
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden", "--expt-relaxed-constexpr",
         "-I", str(CSRC), "-I", str(INCLUDE)]


def sources():
    return sorted(CSRC.glob("*.cu"))


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(p.stat().st_mtime > t for p in deps)


def _compile(src: Path, obj: Path, extra):
    cmd = [NVCC] + ARCH + FLAGS + list(extra) + ["-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src.name, r.stdout[-6000:], r.stderr[-6000:]))
    return r.stderr


def build(force: bool = False, verbose: bool = False, extra=(), stats: bool = False) -> Path:
    """Build libeggsync.so, or with ``stats`` libeggsync_stats.so: the same
    kernels with the update kernel's interaction counters compiled in
    (-DEGG_UPDATE_STATS), for measurement only."""
    objdir = LIBDIR / "stats" if stats else LIBDIR
    lib = LIBDIR / "libeggsync_stats.so" if stats else LIB
    if stats:
        extra = tuple(extra) + ("-DEGG_UPDATE_STATS",)
    objdir.mkdir(parents=True, exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    srcs = sources()
    objs = [objdir / (s.stem + ".o") for s in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _stale(o, [s] + headers)]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            futs = {ex.submit(_compile, s, o, extra): s for s, o in todo}
            for f in cf.as_completed(futs):
                msg = f.result()
                if verbose and msg:
                    sys.stderr.write(msg)
    if force or todo or _stale(lib, objs):
        tmp = lib.with_suffix(".so.tmp%d" % os.getpid())
        # the CUDA runtime is linked statically: the library does not depend
        # on which libcudart the host process (e.g. torch) happens to load
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", str(tmp)] + [str(o) for o in objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (r.stdout[-4000:], r.stderr[-4000:]))
        os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if v else []
    print(build(force="--force" in sys.argv, verbose=v, extra=extra, stats="--stats" in sys.argv))
