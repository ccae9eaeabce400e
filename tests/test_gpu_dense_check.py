"""GPU factor and solve against an independent dense Cholesky (numpy/LAPACK)
of the same permuted matrix, on small inputs."""
import numpy as np
import pytest

from sympack_b200 import DistSparseMatrix, generators as G, symPACKMatrix2D, symPACKOptions

pytestmark = pytest.mark.gpu


def dense_permuted(A: DistSparseMatrix, invp):
    n = A.size
    D = np.zeros((n, n))
    cols = np.repeat(np.arange(n), np.diff(A.colptr))
    rows = A.rowind - 1
    pr, pc = invp[rows] - 1, invp[cols] - 1
    D[pr, pc] = A.nzvalLocal
    D[pc, pr] = A.nzvalLocal
    return D


def factor_as_dense(M: symPACKMatrix2D, n):
    xs = M.GetSupernodalPartition()
    xl, li = M.GetStructure()
    f = M.GetFactor()
    L = np.zeros((n, n))
    pos = 0
    for s in range(len(xs) - 1):
        w = xs[s + 1] - xs[s]
        rows = li[xl[s] - 1:xl[s + 1] - 1] - 1
        h = len(rows)
        panel = f[pos:pos + h * w].reshape(w, h).T
        L[np.ix_(rows, np.arange(xs[s] - 1, xs[s + 1] - 1))] = panel
        pos += h * w
    return L


CASES = [
    ("lap2d_20", lambda: G.laplacian_2d(20, 20)),
    ("lap3d_9", lambda: G.laplacian_3d(9, 9, 9, shift=1e-3)),
    ("st27_7", lambda: G.stencil27(7, 7, 7, 1e-2)),
    ("st27_11", lambda: G.stencil27(11, 11, 11, 1e-2)),
    ("rand_900", lambda: G.random_graph_spd(900, 10, 1.05, seed=3)),
]


@pytest.mark.parametrize("name,gen", CASES)
def test_factor_matches_dense_cholesky(name, gen):
    n, cp, ri, v = gen()
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions())
    M.SymbolicFactorization(A)
    M.DistributeMatrix(A)
    M.Factorize()
    perm, invp = M.GetOrdering()
    D = dense_permuted(A, invp)
    Lref = np.linalg.cholesky(D)
    L = factor_as_dense(M, n)
    assert np.max(np.abs(L - Lref)) <= 1e-12 * np.max(np.abs(Lref))
    rng = np.random.default_rng(0)
    for nrhs in (1, 5):
        b = rng.uniform(-1, 1, size=(n, nrhs))
        M.Solve(b)
        x = M.GetSolution(nrhs=nrhs)
        Afull = D[np.ix_(invp - 1, invp - 1)]
        xref = np.linalg.solve(Afull, b)
        assert np.max(np.abs(x - xref)) <= 1e-12 * np.max(np.abs(xref))
