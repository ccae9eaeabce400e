"""ORACLE build recipe: compile numeric_oracle.c into oracle/_build/liboracle.so,
linked against scipy's bundled OpenBLAS (exported scipy_d*_ names)."""
from __future__ import annotations

import glob
import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build" / "liboracle.so"


def openblas_lib() -> Path:
    import scipy
    libdir = Path(scipy.__file__).resolve().parent.parent / "scipy.libs"
    cands = sorted(glob.glob(str(libdir / "libscipy_openblas*.so")))
    if not cands:
        raise RuntimeError(f"scipy's bundled OpenBLAS not found under {libdir}")
    return Path(cands[0])


def needs_build() -> bool:
    src = HERE / "numeric_oracle.c"
    return not OUT.exists() or src.stat().st_mtime > OUT.stat().st_mtime


def build(force: bool = False) -> Path:
    if not force and not needs_build():
        return OUT
    OUT.parent.mkdir(exist_ok=True)
    blas = openblas_lib()
    tmp = OUT.with_suffix(".tmp.so")
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-o", str(tmp), str(HERE / "numeric_oracle.c"),
           str(blas), f"-Wl,-rpath,{blas.parent}", "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True))
