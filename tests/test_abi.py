"""The C-ABI library loads and exports every entry point include/*.h declares;
host-only handles give the documented status codes (no GPU needed)."""
import glob
import os
import re

import numpy as np
import pytest

from sympack_b200 import DistSparseMatrix, StateError, generators as G, symPACKMatrix2D, symPACKOptions
from sympack_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names.update(re.findall(r"\b(spb_\w+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = N.load()
    decl = declared_symbols()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(lib, name), name
    assert set(N.exported_symbols()) >= set(decl)


def test_host_only_handle_rejects_numeric_calls():
    n, cp, ri, v = G.laplacian_2d(8, 8)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1))
    M.SymbolicFactorization(A)
    for call in (lambda: M.DistributeMatrix(A), M.Factorize, lambda: M.Solve(np.ones(n))):
        with pytest.raises(StateError):
            call()


def test_calls_out_of_order():
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1))
    with pytest.raises(StateError):
        M.info()


def test_bad_options():
    with pytest.raises(ValueError):
        symPACKMatrix2D().Init(symPACKOptions(orderingStr="METIS"))
    with pytest.raises(ValueError):
        symPACKMatrix2D().Init(symPACKOptions(orderingStr="USER"))
