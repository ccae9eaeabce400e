"""ORACLE — ctypes wrapper of numeric_oracle.c (CPU restatement of the
reference's 2D numeric path).  Test / baseline infrastructure only."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import build_oracle

_lib = None


def load():
    global _lib
    if _lib is None:
        build_oracle.build()
        lib = C.CDLL(str(build_oracle.OUT))
        I32P, I64P, DP, VP = C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_double), C.c_void_p
        lib.orc_create.restype = VP
        lib.orc_create.argtypes = [C.c_int, C.c_int, I32P, I64P, I32P, I32P, I32P]
        lib.orc_destroy.argtypes = [VP]
        lib.orc_distribute.argtypes = [VP, I64P, I32P, DP]
        lib.orc_factorize.argtypes = [VP]
        lib.orc_solve.argtypes = [VP, DP, C.c_int, C.c_int64]
        lib.orc_get_factor.argtypes = [VP, DP]
        lib.orc_status.argtypes = [VP]
        lib.orc_set_threads.argtypes = [C.c_int]
        lib.orc_set_ldl.argtypes = [VP, C.c_int]
        _lib = lib
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class OracleFactor:
    """One factorization: cells built from a symbolic result (dict of arrays);
    ldl=True runs the reference's LDL^T cells (D on the factor's diagonal)."""

    def __init__(self, n, sym, threads=None, ldl=False):
        lib = load()
        if threads:
            lib.orc_set_threads(int(threads))
        self.n = n
        self._keep = [np.ascontiguousarray(sym["xsuper"], np.int32), np.ascontiguousarray(sym["xlindx"], np.int64),
                      np.ascontiguousarray(sym["lindx"], np.int32), np.ascontiguousarray(sym["supmember"], np.int32),
                      np.ascontiguousarray(sym["invp"], np.int32)]
        xs, xl, li, sm, iv = self._keep
        self.nsuper = len(xs) - 1
        self.h = lib.orc_create(n, self.nsuper, _p(xs, C.c_int32), _p(xl, C.c_int64), _p(li, C.c_int32),
                                _p(sm, C.c_int32), _p(iv, C.c_int32))
        self.factor_size = int(np.sum((xl[1:] - xl[:-1]) * (xs[1:] - xs[:-1])))
        if ldl:
            lib.orc_set_ldl(self.h, 1)

    def distribute(self, colptr, rowind, nzval):
        cp = np.ascontiguousarray(colptr, np.int64)
        ri = np.ascontiguousarray(rowind, np.int32)
        v = np.ascontiguousarray(nzval, np.float64)
        rc = load().orc_distribute(self.h, _p(cp, C.c_int64), _p(ri, C.c_int32), _p(v, C.c_double))
        if rc:
            raise RuntimeError(f"oracle distribute failed ({rc})")

    def factorize(self):
        rc = load().orc_factorize(self.h)
        if rc == -2:
            raise ArithmeticError(f"Matrix is not HPD / zero pivot (supernode {load().orc_status(self.h)})")
        if rc:
            raise RuntimeError(f"oracle factorize failed ({rc})")

    def solve(self, B):
        X = np.asfortranarray(np.array(B, dtype=np.float64).reshape(self.n, -1, order="F"))
        rc = load().orc_solve(self.h, _p(X, C.c_double), X.shape[1], self.n)
        if rc:
            raise RuntimeError(f"oracle solve failed ({rc})")
        return X.reshape(np.shape(B), order="F") if np.ndim(B) == 1 else X

    def factor(self):
        out = np.empty(self.factor_size, np.float64)
        load().orc_get_factor(self.h, _p(out, C.c_double))
        return out

    def __del__(self):
        try:
            if self.h:
                load().orc_destroy(self.h)
                self.h = None
        except Exception:
            pass
