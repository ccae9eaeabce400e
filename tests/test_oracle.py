"""The numeric oracle (C restatement of the reference's cell algorithm) pinned
against numpy/LAPACK dense Cholesky and solve on the same permuted matrix."""
import numpy as np
import pytest

from oracle import numeric, symbolic_oracle as so
from sympack_b200 import DistSparseMatrix, generators as G

CASES = [
    ("lap2d_64", lambda: G.laplacian_2d(64, 64)),
    ("lap3d_10", lambda: G.laplacian_3d(10, 10, 10, 1e-3)),
    ("st27_8", lambda: G.stencil27(8, 8, 8, 1e-2)),
    ("rand_800", lambda: G.random_graph_spd(800, 10, 1.05, seed=4)),
]


def dense_from_factor(fac, sym, n):
    xs, xl, li = sym["xsuper"], sym["xlindx"], sym["lindx"]
    L = np.zeros((n, n))
    pos = 0
    for s in range(len(xs) - 1):
        w = xs[s + 1] - xs[s]
        rows = li[xl[s] - 1:xl[s + 1] - 1] - 1
        h = len(rows)
        L[np.ix_(rows, np.arange(xs[s] - 1, xs[s + 1] - 1))] = fac[pos:pos + h * w].reshape(w, h).T
        pos += h * w
    return L


@pytest.mark.parametrize("name,gen", CASES)
def test_oracle_factor_and_solve_match_lapack(name, gen):
    n, cp, ri, v = gen()
    sym = so.symbolic_chain(n, cp, ri)
    f = numeric.OracleFactor(n, sym, threads=2)
    f.distribute(cp, ri, v)
    f.factorize()
    invp = sym["invp"]
    D = np.zeros((n, n))
    cols = np.repeat(np.arange(n), np.diff(cp))
    D[invp[ri - 1] - 1, invp[cols] - 1] = v
    D[invp[cols] - 1, invp[ri - 1] - 1] = v
    Lref = np.linalg.cholesky(D)
    L = dense_from_factor(f.factor(), sym, n)
    assert np.max(np.abs(L - Lref)) <= 1e-13 * np.max(np.abs(Lref))
    rng = np.random.default_rng(1)
    B = rng.standard_normal((n, 3))
    X = f.solve(B)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    assert np.linalg.norm(A.matvec(X) - B) / np.linalg.norm(B) < 1e-13


def test_oracle_detects_non_spd():
    n, cp, ri, v = G.laplacian_2d(10, 10)
    v = v.copy()
    v[cp[37] - 1] = -5.0  # diagonal of column 38
    sym = so.symbolic_chain(n, cp, ri)
    f = numeric.OracleFactor(n, sym)
    f.distribute(cp, ri, v)
    with pytest.raises(ArithmeticError):
        f.factorize()
