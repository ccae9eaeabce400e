"""DumpMatlab and the symPACKMatrixMeta accessors (symPACKMatrixBase.hpp:96-103,
2D.hpp:6762-6854) on the host: the MATLAB text of a factor (the CPU oracle's, in the
library's panel layout) read back equals the dense Cholesky factor of the permuted matrix;
Size / TotalSupernodeCnt / GetOptions on an analysed host-only handle."""
import io
import re

import numpy as np

from oracle import numeric
from sympack_b200 import DistSparseMatrix, generators as G, symPACKMatrix2D, symPACKOptions
from sympack_b200.solver import matlab_sparse


def _analyse(n, cp, ri, v, **opt):
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1, **opt))
    M.SymbolicFactorization(DistSparseMatrix.from_lower_csc(n, cp, ri, v))
    return M


def _read_matlab(text):
    m = re.fullmatch(r"\+sparse\(\[([^\]]*)\],\[([^\]]*)\],\[([^\]]*)\],(\d+),(\d+)\)\n", text)
    assert m, text[:200]
    rows = np.array(m.group(1).split(), np.int64)
    cols = np.array(m.group(2).split(), np.int64)
    vals = np.array(m.group(3).split(), np.float64)
    n = int(m.group(4))
    assert int(m.group(5)) == n and len(rows) == len(cols) == len(vals)
    return n, rows, cols, vals


def test_matlab_text_of_the_oracle_factor_is_the_dense_cholesky_factor():
    n, cp, ri, v = G.laplacian_3d(7, 6, 5, 1e-2)
    M = _analyse(n, cp, ri, v)
    perm, invp = M.GetOrdering()
    xs = M.GetSupernodalPartition()
    xl, li = M.GetStructure()
    sym = dict(xsuper=xs, xlindx=xl, lindx=li, supmember=M.GetSupMembership(), invp=invp)
    f = numeric.OracleFactor(n, sym, threads=2)
    f.distribute(cp, ri, v)
    f.factorize()
    text = matlab_sparse(n, xs, xl, li, f.factor())
    nn, rows, cols, vals = _read_matlab(text)
    assert nn == n
    assert np.all(rows >= cols) and rows.min() >= 1 and rows.max() <= n
    assert len(set(zip(rows.tolist(), cols.tolist()))) == len(rows)  # each entry once
    # stored entries: the lower triangle of every supernode's panel
    w = np.diff(xs)
    h = np.diff(xl)
    assert len(rows) == int(np.sum(w * h - w * (w - 1) // 2))
    L = np.zeros((n, n))
    L[rows - 1, cols - 1] = vals
    A = np.zeros((n, n))
    colidx = np.repeat(np.arange(n), np.diff(cp))
    A[ri - 1, colidx] = v
    A = A + np.tril(A, -1).T
    Ap = np.empty_like(A)
    Ap[np.ix_(invp - 1, invp - 1)] = A  # row/column i of A is row/column invp[i] of the permuted matrix
    np.testing.assert_allclose(L, np.linalg.cholesky(Ap), rtol=0, atol=1e-13)
    # supernode by supernode, row by row: the first entries are the first supernode's first row
    assert rows[0] == xs[0] and cols[0] == xs[0]


def test_accessors_and_dump_to_a_stream():
    n, cp, ri, v = G.laplacian_2d(9, 8, 1e-3)
    opts = symPACKOptions(device=-1, orderingStr="AMD")
    M = symPACKMatrix2D()
    assert M.Size() == 0
    M.Init(opts)
    assert M.GetOptions() is opts and M.TotalSupernodeCnt() == 0
    M.SymbolicFactorization(DistSparseMatrix.from_lower_csc(n, cp, ri, v))
    assert M.Size() == n
    assert M.TotalSupernodeCnt() == len(M.GetSupernodalPartition()) - 1 == M.info().nsuper
    # the text of a made-up factor (value = 1000 row + column) through a stream
    xs = M.GetSupernodalPartition()
    xl, li = M.GetStructure()
    panels = []
    for s in range(len(xs) - 1):
        r = li[xl[s] - 1:xl[s + 1] - 1].astype(np.float64)
        c = np.arange(xs[s], xs[s + 1], dtype=np.float64)
        panels.append((1000.0 * r[:, None] + c[None, :]).T.ravel())  # column-major h x w
    buf = io.StringIO()
    buf.write(matlab_sparse(n, xs, xl, li, np.concatenate(panels)))
    _, rows, cols, vals = _read_matlab(buf.getvalue())
    np.testing.assert_array_equal(vals, 1000.0 * rows + cols)
    M.close()
