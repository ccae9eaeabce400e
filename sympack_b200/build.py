"""Build the native library of the package in-tree.

    python -m sympack_b200.build          # builds sympack_b200/_lib/libsympack_b200.so

All CUDA code is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``).
The library is rebuilt when any source under ``csrc/`` or ``include/`` is newer
than it.
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
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "libsympack_b200.so"

SOURCES = ["symbolic.cpp", "amd.cpp", "plan.cpp", "rb_io.cpp", "kernels.cu", "gemm.cu", "solve.cu", "ir.cu", "capi.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build sympack_b200")


def _inputs() -> list[Path]:
    files = [CSRC / s for s in SOURCES]
    files += sorted(CSRC.glob("*.hpp")) + sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))
    return files


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(f.stat().st_mtime > t for f in _inputs() if f.exists())


def build(verbose: bool = False, force: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    LIBDIR.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objdir = LIBDIR / "obj"
    objdir.mkdir(exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo", "-I", str(ROOT / "include")]
    for src in SOURCES:
        obj = objdir / (src + ".o")
        cmd = [nvcc, *common, *ARCH, "-c", str(CSRC / src), "-o", str(obj)]
        if src.endswith(".cu"):
            cmd[1:1] = ["-Xptxas", "-v"] if verbose else []
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, "-shared", *ARCH, "-o", str(tmp), *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
