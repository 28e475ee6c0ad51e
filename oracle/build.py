"""Build recipe for the oracle (test infrastructure only).

* ``build_oracle()`` compiles the C restatement ``oracle/egg_oracle.c`` into
  ``oracle/_build/libeggoracle.so``.
* ``build_ref()`` compiles the reference's own sources, where they lie in
  the reference tree (its location comes from the ``root`` argument or the
  ``EGG_REFERENCE_ROOT`` environment variable; never copied), together with the two thin C-ABI
  drivers in this folder, into ``oracle/_ref/``:

  - ``libref_sync.so``: ``src/algorithms/SynC.cpp`` + ``src/utils/CPU_math.cpp``
    + ``ref_sync_driver.cpp`` (the reference CPU SynC, OpenMP).
  - ``libref_egg.so``: ``src/algorithms/EGG_SynC.cu`` + ``src/utils/GPU_utils.cu``
    + ``src/utils/CPU_math.cpp`` + ``ref_egg_driver.cu`` (the reference
    EGG-SynC, sm_100a).

  Three flag changes against ``python/algorithms.py:6-17`` are needed with
  this toolchain: ``--std=c++17`` (torch 2.11 headers), ``-include cstdio``
  (``CPU_math.cpp`` uses printf without including it) and an explicit
  ``-fopenmp``/libgomp link.  The reference's own build (a torch JIT
  ``load``) is not run.

The outputs are git-ignored but travel with copies of the working tree, so a
machine without the reference tree uses the files built here.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
BUILD_DIR = HERE / "_build"
REF_DIR = HERE / "_ref"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s\n%s" % (" ".join(map(str, cmd)), r.stdout[-4000:], r.stderr[-4000:]))
    return r


def oracle_lib_path() -> Path:
    return BUILD_DIR / "libeggoracle.so"


def build_oracle(force: bool = False) -> Path:
    out = oracle_lib_path()
    src = HERE / "egg_oracle.c"
    if out.exists() and not force and out.stat().st_mtime >= src.stat().st_mtime:
        return out
    BUILD_DIR.mkdir(exist_ok=True)
    tmp = out.with_suffix(".so.tmp%d" % os.getpid())
    _run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", str(src), "-o", str(tmp), "-lm"])
    os.replace(tmp, out)
    return out


def _torch_flags():
    import torch
    from torch.utils import cpp_extension as ce

    inc = []
    for p in ce.include_paths():
        inc += ["-I", p]
    libdir = os.path.join(os.path.dirname(torch.__file__), "lib")
    abi = "-D_GLIBCXX_USE_CXX11_ABI=%d" % int(torch._C._GLIBCXX_USE_CXX11_ABI)
    link = ["-L" + libdir, "-Wl,-rpath," + libdir, "-lc10", "-ltorch_cpu", "-ltorch"]
    return inc, abi, link


def ref_root(root=None):
    """The reference tree: ``root`` if given, else ``EGG_REFERENCE_ROOT``, else None."""
    r = root if root is not None else os.environ.get("EGG_REFERENCE_ROOT")
    return Path(r) if r else None


def ref_available(root=None) -> bool:
    r = ref_root(root)
    return r is not None and (r / "src" / "algorithms" / "SynC.cpp").exists()


def build_ref(force: bool = False, with_gpu: bool = True, root=None) -> dict:
    """Compile the reference CPU SynC (and, with ``with_gpu``, EGG-SynC and the
    brute-force GPU SynC) from the reference tree ``root`` (default:
    ``EGG_REFERENCE_ROOT``)."""
    if not ref_available(root):
        raise FileNotFoundError("reference sources not found (give root= or set EGG_REFERENCE_ROOT)")
    REF_DIR.mkdir(exist_ok=True)
    inc, abi, link = _torch_flags()
    src = ref_root(root) / "src"
    out = {}

    sync_so = REF_DIR / "libref_sync.so"
    if force or not sync_so.exists():
        objs = []
        for f in [src / "algorithms" / "SynC.cpp", src / "utils" / "CPU_math.cpp", HERE / "ref_sync_driver.cpp"]:
            o = REF_DIR / (f.stem + ".sync.o")
            _run(["g++", "-O3", "-fPIC", "-std=c++17", "-w", "-fopenmp", "-include", "cstdio", abi,
                  "-I", str(src / "algorithms"), "-I", str(src / "utils")] + inc + ["-c", str(f), "-o", str(o)])
            objs.append(str(o))
        tmp = sync_so.with_suffix(".so.tmp")
        _run(["g++", "-shared", "-fopenmp", "-o", str(tmp)] + objs + link + ["-lgomp"])
        os.replace(tmp, sync_so)
    out["sync"] = sync_so

    if with_gpu:
        egg_so = REF_DIR / "libref_egg.so"
        if force or not egg_so.exists():
            objs = []
            cu = [src / "algorithms" / "EGG_SynC.cu", src / "utils" / "GPU_utils.cu", HERE / "ref_egg_driver.cu"]
            for f in cu:
                o = REF_DIR / (f.stem + ".egg.o")
                _run(["nvcc", "-O3", "-std=c++17", "-w", "-Xcompiler", "-fPIC", abi] + ARCH +
                     ["-I", str(src / "algorithms"), "-I", str(src / "utils")] + inc + ["-c", str(f), "-o", str(o)])
                objs.append(str(o))
            o = REF_DIR / "CPU_math.egg.o"
            _run(["g++", "-O3", "-fPIC", "-std=c++17", "-w", "-include", "cstdio", abi] + inc +
                 ["-c", str(src / "utils" / "CPU_math.cpp"), "-o", str(o)])
            objs.append(str(o))
            tmp = egg_so.with_suffix(".so.tmp")
            _run(["nvcc", "-shared", "-Xcompiler", "-fPIC", "-o", str(tmp)] + objs +
                 ["-Xlinker", "-rpath," + link[0][2:]] + [x for x in link if not x.startswith("-Wl")] + ["-lcudart"])
            os.replace(tmp, egg_so)
        out["egg"] = egg_so
        simple_so = REF_DIR / "libref_simple.so"
        if force or not simple_so.exists():
            objs = []
            cu = [src / "algorithms" / "simple_GPU_SynC.cu", src / "utils" / "GPU_utils.cu",
                  HERE / "ref_simple_driver.cu"]
            for f in cu:
                o = REF_DIR / (f.stem + ".simple.o")
                _run(["nvcc", "-O3", "-std=c++17", "-w", "-Xcompiler", "-fPIC", abi] + ARCH +
                     ["-I", str(src / "algorithms"), "-I", str(src / "utils")] + inc + ["-c", str(f), "-o", str(o)])
                objs.append(str(o))
            o = REF_DIR / "CPU_math.simple.o"
            _run(["g++", "-O3", "-fPIC", "-std=c++17", "-w", "-include", "cstdio", abi] + inc +
                 ["-c", str(src / "utils" / "CPU_math.cpp"), "-o", str(o)])
            objs.append(str(o))
            tmp = simple_so.with_suffix(".so.tmp")
            _run(["nvcc", "-shared", "-Xcompiler", "-fPIC", "-o", str(tmp)] + objs +
                 ["-Xlinker", "-rpath," + link[0][2:]] + [x for x in link if not x.startswith("-Wl")] + ["-lcudart"])
            os.replace(tmp, simple_so)
        out["simple"] = simple_so
    return out


if __name__ == "__main__":
    # python oracle/build.py [--force] [--no-gpu] [--ref REFERENCE_TREE]
    print(build_oracle(force="--force" in sys.argv))
    root = sys.argv[sys.argv.index("--ref") + 1] if "--ref" in sys.argv else None
    if ref_available(root):
        print(build_ref(force="--force" in sys.argv, with_gpu="--no-gpu" not in sys.argv, root=root))
