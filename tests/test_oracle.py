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


def dense_ldl(D):
    """Unpivoted dense LDL^T (column by column), the reference's Potf2_LDL recurrence."""
    n = D.shape[0]
    A = D.copy()
    L, d = np.eye(n), np.zeros(n)
    for k in range(n):
        d[k] = A[k, k]
        L[k + 1:, k] = A[k + 1:, k] / d[k]
        A[k + 1:, k + 1:] -= np.outer(L[k + 1:, k], A[k, k + 1:])
    return L, d


@pytest.mark.parametrize("name,gen", [("qd_8", lambda: G.quasi_definite_3d(8, 8, 8, 0.3, 1e-2, seed=1)),
                                      ("qd_6x9x5", lambda: G.quasi_definite_3d(6, 9, 5, 0.5, 1e-2, seed=2)),
                                      ("st27_8_spd", lambda: G.stencil27(8, 8, 8, 1e-2))])
def test_oracle_ldl_matches_dense_ldl(name, gen):
    """The LDL^T oracle (D on the factor's diagonal, unit L below) against a dense
    unpivoted LDL^T of the same permuted matrix, and its solve against the matrix."""
    n, cp, ri, v = gen()
    sym = so.symbolic_chain(n, cp, ri)
    f = numeric.OracleFactor(n, sym, threads=2, ldl=True)
    f.distribute(cp, ri, v)
    f.factorize()
    invp = sym["invp"]
    cols = np.repeat(np.arange(n), np.diff(cp))
    D = np.zeros((n, n))
    D[invp[ri - 1] - 1, invp[cols] - 1] = v
    D[invp[cols] - 1, invp[ri - 1] - 1] = v
    Lref, dref = dense_ldl(D)
    F = dense_from_factor(f.factor(), sym, n)
    assert np.max(np.abs(np.diag(F) - dref)) <= 1e-12 * np.max(np.abs(dref))
    Lo = np.tril(F, -1) + np.eye(n)
    assert np.max(np.abs(Lo - Lref)) <= 1e-12 * np.max(np.abs(Lref))
    B = np.random.default_rng(3).standard_normal((n, 2))
    X = f.solve(B)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    assert np.linalg.norm(A.matvec(X) - B) / np.linalg.norm(B) < 1e-12


def test_quasi_definite_generator_structure():
    """[H B^T; B -G] with H and G strictly diagonally dominant over their own block."""
    n, cp, ri, v = G.quasi_definite_3d(7, 6, 5, 0.4, 1e-2, seed=9)
    cols = np.repeat(np.arange(n), np.diff(cp))
    rows = ri - 1
    diag = v[cp[:-1] - 1]
    assert np.all(rows[cp[:-1] - 1] == np.arange(n))  # first entry of each column is its diagonal
    sign = np.sign(diag)
    assert set(np.unique(sign)) == {-1.0, 1.0}
    same = (sign[rows] == sign[cols]) & (rows != cols)
    dom = np.zeros(n)
    np.add.at(dom, rows[same], np.abs(v[same]))
    np.add.at(dom, cols[same], np.abs(v[same]))
    assert np.all(np.abs(diag) > dom)
