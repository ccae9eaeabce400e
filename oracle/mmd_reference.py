"""ORACLE — the reference's own MMD Fortran (src/ordmmd.F, genmmd.F, mmdint.F,
mmdelm.F, mmdupd.F, mmdnum.F), RCM Fortran (src/genrcm.F, rcm.F, fnroot.F,
rootls.F, degree.F) and AMD Fortran (src/amdbar.F), translated by
oracle/f77_to_c.py and compiled into oracle/_ref/libmmd_ref.so,
oracle/_ref/librcm_ref.so and oracle/_ref/libamd_ref.so.  Building needs the reference sources
(present in the development container only); the built library may travel.
Called exactly as Ordering::MMD calls it (src/Ordering.cpp:103-218): the
expanded graph without diagonal, iwsiz = 4n, invp taken as the result."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# Reference source tree: $SYMPACK_REFERENCE (the symPACK checkout), default /root/reference.
REF_ROOT = Path(os.environ.get("SYMPACK_REFERENCE", "/root/reference"))
REF_SRC = REF_ROOT / "src"
FILES = ["ordmmd.F", "genmmd.F", "mmdint.F", "mmdelm.F", "mmdupd.F", "mmdnum.F"]
OUT_C = HERE / "_ref" / "mmd_ref.c"
OUT_SO = HERE / "_ref" / "libmmd_ref.so"
_lib = None


def available() -> bool:
    return OUT_SO.exists() or all((REF_SRC / f).exists() for f in FILES)


def build(force: bool = False) -> Path:
    if OUT_SO.exists() and not force:
        return OUT_SO
    if not all((REF_SRC / f).exists() for f in FILES):
        raise FileNotFoundError("reference MMD sources not present")
    OUT_SO.parent.mkdir(exist_ok=True)
    from . import f77_to_c
    OUT_C.write_text(f77_to_c.translate([str(REF_SRC / f) for f in FILES]))
    tmp = OUT_SO.with_suffix(".tmp.so")
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-Wno-unused-label", "-o", str(tmp), str(OUT_C)], check=True)
    os.replace(tmp, OUT_SO)
    return OUT_SO


def ordmmd(n: int, xadj, adj) -> np.ndarray:
    """invp (1-based) of the reference MMD on a graph given as 1-based xadj/adj."""
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(build()))
    P = C.POINTER(C.c_int32)
    xadj = np.ascontiguousarray(xadj, np.int32)
    adj = np.ascontiguousarray(adj, np.int32).copy()  # destroyed by genmmd
    invp = np.zeros(n, np.int32)
    perm = np.zeros(n, np.int32)
    iwsiz = C.c_int32(4 * n)
    iwork = np.zeros(4 * n, np.int32)
    N, nadj, nofsub, iflag = C.c_int32(n), C.c_int32(len(adj)), C.c_int32(0), C.c_int32(0)
    _lib.ordmmd_(C.byref(N), C.byref(nadj), xadj.ctypes.data_as(P), adj.ctypes.data_as(P),
                 invp.ctypes.data_as(P), perm.ctypes.data_as(P), C.byref(iwsiz), iwork.ctypes.data_as(P),
                 C.byref(nofsub), C.byref(iflag))
    if iflag.value != 0:
        raise RuntimeError(f"ordmmd iflag={iflag.value}")
    return invp


RCM_FILES = ["genrcm.F", "rcm.F", "fnroot.F", "rootls.F", "degree.F"]
OUT_RCM_C = HERE / "_ref" / "rcm_ref.c"
OUT_RCM_SO = HERE / "_ref" / "librcm_ref.so"
_rcm = None


def rcm_available() -> bool:
    return OUT_RCM_SO.exists() or all((REF_SRC / f).exists() for f in RCM_FILES)


def build_rcm(force: bool = False) -> Path:
    if OUT_RCM_SO.exists() and not force:
        return OUT_RCM_SO
    if not all((REF_SRC / f).exists() for f in RCM_FILES):
        raise FileNotFoundError("reference RCM sources not present")
    OUT_RCM_SO.parent.mkdir(exist_ok=True)
    from . import f77_to_c
    OUT_RCM_C.write_text(f77_to_c.translate([str(REF_SRC / f) for f in RCM_FILES]))
    tmp = OUT_RCM_SO.with_suffix(".tmp.so")
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-Wno-unused-label", "-Wno-unused-function", "-o", str(tmp),
                    str(OUT_RCM_C)], check=True)
    os.replace(tmp, OUT_RCM_SO)
    return OUT_RCM_SO


def genrcm(n: int, xadj, adj) -> np.ndarray:
    """invp (1-based) of the reference RCM, called as Ordering::RCM calls it
    (src/Ordering.cpp:221-300): expanded graph without diagonal, mark and xls of
    size 2n, invp[perm[i]] = i."""
    global _rcm
    if _rcm is None:
        _rcm = C.CDLL(str(build_rcm()))
    P = C.POINTER(C.c_int32)
    xadj = np.ascontiguousarray(xadj, np.int32).copy()  # DEGREE flips signs and restores them
    adj = np.ascontiguousarray(adj, np.int32)
    perm = np.zeros(n, np.int32)
    mark = np.zeros(2 * n, np.int32)
    xls = np.zeros(2 * n, np.int32)
    N = C.c_int32(n)
    _rcm.genrcm_(C.byref(N), xadj.ctypes.data_as(P), adj.ctypes.data_as(P), perm.ctypes.data_as(P),
                 mark.ctypes.data_as(P), xls.ctypes.data_as(P))
    invp = np.zeros(n, np.int32)
    invp[perm - 1] = np.arange(1, n + 1, dtype=np.int32)
    return invp


AMD_FILES = ["amdbar.F"]
OUT_AMD_C = HERE / "_ref" / "amd_ref.c"
OUT_AMD_SO = HERE / "_ref" / "libamd_ref.so"
_amd = None


def amd_available() -> bool:
    return OUT_AMD_SO.exists() or all((REF_SRC / f).exists() for f in AMD_FILES)


def build_amd(force: bool = False) -> Path:
    if OUT_AMD_SO.exists() and not force:
        return OUT_AMD_SO
    if not all((REF_SRC / f).exists() for f in AMD_FILES):
        raise FileNotFoundError("reference AMD sources not present")
    OUT_AMD_SO.parent.mkdir(exist_ok=True)
    from . import f77_to_c
    OUT_AMD_C.write_text(f77_to_c.translate([str(REF_SRC / f) for f in AMD_FILES]))
    tmp = OUT_AMD_SO.with_suffix(".tmp.so")
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-Wno-unused-label", "-Wno-unused-function",
                    "-fwrapv", "-o", str(tmp), str(OUT_AMD_C)], check=True)
    os.replace(tmp, OUT_AMD_SO)
    return OUT_AMD_SO


def amdbar(n: int, xadj, adj) -> np.ndarray:
    """invp (1-based) of the reference AMD, called as Ordering::AMD calls it
    (src/Ordering.cpp:411-520): expanded graph without diagonal, IW of nnz + n
    entries, IWLEN = nnz + n, PFREE = nnz + 1, IOVFLO = INT32_MAX; ELEN is invp."""
    global _amd
    if _amd is None:
        _amd = C.CDLL(str(build_amd()))
    P = C.POINTER(C.c_int32)
    nnz = len(adj)
    pe = np.ascontiguousarray(xadj, np.int32)[:n + 1].copy()
    iw = np.zeros(nnz + n, np.int32)
    iw[:nnz] = adj
    ln = np.diff(np.ascontiguousarray(xadj, np.int64)).astype(np.int32)
    ln = np.append(ln, 0).astype(np.int32)
    qsize, ecforw, perm, marker, vtxdeg, invp = (np.zeros(n, np.int32) for _ in range(6))
    iwork = np.zeros(4 * n, np.int32)
    N, iwlen, pfree = C.c_int32(n), C.c_int32(nnz + n), C.c_int32(nnz + 1)
    ncmpa, iovflo = C.c_int32(0), C.c_int32(2 ** 31 - 1)
    _amd.amdbar_(C.byref(N), pe.ctypes.data_as(P), iw.ctypes.data_as(P), ln.ctypes.data_as(P), C.byref(iwlen),
                 C.byref(pfree), qsize.ctypes.data_as(P), ecforw.ctypes.data_as(P), perm.ctypes.data_as(P),
                 iwork.ctypes.data_as(P), invp.ctypes.data_as(P), vtxdeg.ctypes.data_as(P), C.byref(ncmpa),
                 marker.ctypes.data_as(P), C.byref(iovflo))
    return invp
