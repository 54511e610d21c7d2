"""Build the native library libthesiscode_b200.so in-tree for sm_100a.

Every CUDA and C++ source under ``csrc/`` is compiled by nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and linked into
``thesiscode_b200/_lib/libthesiscode_b200.so``. The library has no torch
types in its ABI and links only the CUDA runtime, so a C, C++ or Fortran
caller can load it directly. Objects are rebuilt only when a source or
header is newer than the library.

``--checked`` builds the same sources with ``-DTC_BOUNDS_CHECK=1`` into
``libthesiscode_b200_checked.so``: its hot-path kernels check every
global-memory index against its array's extent and record violations
(tc_bounds_status) instead of accessing out of range. ``TC_LIBRARY=checked``
makes the Python package load it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIBDIR = PKG / "_lib"
LIBNAME = "libthesiscode_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "-Xptxas", "-O3",
]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the sm_100a library cannot be built")


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


CHECKED_LIBNAME = "libthesiscode_b200_checked.so"


def lib_path(checked: bool = False) -> Path:
    return LIBDIR / (CHECKED_LIBNAME if checked else LIBNAME)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, checked: bool = False) -> Path:
    """Compile csrc/ into _lib/libthesiscode_b200.so (checked: the index-checked
    libthesiscode_b200_checked.so); returns the library path."""
    nvcc = nvcc_path()
    objdir = LIBDIR / ("obj_checked" if checked else "obj")
    defines = ["-DTC_BOUNDS_CHECK=1"] if checked else []
    objdir.mkdir(parents=True, exist_ok=True)
    hdrs = headers()
    objs, cmds = [], []
    for src in sources():
        obj = objdir / (src.name + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            cmds.append([nvcc, *ARCH, *NVCC_FLAGS, *defines, f"-I{INCLUDE}", f"-I{CSRC}", "-c",
                         str(src), "-o", str(obj)])
    # translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor

    def run(cmd):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(run, c) for c in cmds]:
            f.result()
    lib = lib_path(checked)
    if force or _stale(lib, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", str(lib), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv, checked="--checked" in sys.argv))
