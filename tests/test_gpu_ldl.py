"""LDL^T decomposition (DecompositionType::LDL, the reference driver's -fact LDL) on the
GPU against the CPU oracle's restatement of the reference's blockCellLDL_t path, through
the C ABI.  Tolerance 1e-12 relative (max-norm) for the factor (L with D on the
diagonal) and the solution, as for the Cholesky path.  Indefinite cases are
quasi-definite matrices [H B^T; B -G] (H, G diagonally dominant), which have an
LDL^T factorization without pivoting in every ordering."""
import os

import numpy as np
import pytest

from oracle import numeric
from sympack_b200 import DistSparseMatrix, NotSPDError, generators as G, symPACKMatrix2D, symPACKOptions

pytestmark = pytest.mark.gpu
TOL = 1e-12


def setup(A, **opt):
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0, decomposition="LDL", **opt))
    M.SymbolicFactorization(A)
    M.DistributeMatrix(A)
    M.Factorize()
    return M


def oracle_for(M, A):
    perm, invp = M.GetOrdering()
    xl, li = M.GetStructure()
    sym = dict(xsuper=M.GetSupernodalPartition(), xlindx=xl, lindx=li, supmember=M.GetSupMembership(), invp=invp)
    f = numeric.OracleFactor(A.size, sym, threads=os.cpu_count(), ldl=True)
    f.distribute(A.colptr, A.rowind, A.nzvalLocal)
    f.factorize()
    return f


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def diag_of_factor(M):
    """D as stored on the diagonal of the dumped factor (per supernode, h x w column-major)."""
    xs = M.GetSupernodalPartition()
    xl, _ = M.GetStructure()
    fac = M.GetFactor()
    d, pos = [], 0
    for s in range(len(xs) - 1):
        w, h = xs[s + 1] - xs[s], xl[s + 1] - xl[s]
        blk = fac[pos:pos + h * w].reshape(w, h)
        d.extend(blk[j, j] for j in range(w))
        pos += h * w
    return np.array(d)


CASES = [
    ("lap3d_20_spd", lambda: G.laplacian_3d(20, 20, 20, 1e-3), {}),
    ("st27_14_spd", lambda: G.stencil27(14, 14, 14, 1e-2, seed=1), {}),
    ("rand_3000_spd", lambda: G.random_graph_spd(3000, 10, 1.05, seed=9), {}),
    ("qd_16_30pct", lambda: G.quasi_definite_3d(16, 16, 16, 0.3, 1e-2, seed=1), {}),
    ("qd_22_50pct", lambda: G.quasi_definite_3d(22, 22, 22, 0.5, 1e-2, seed=2), {}),
    ("qd_12_amd", lambda: G.quasi_definite_3d(12, 12, 12, 0.4, 1e-2, seed=3), {"orderingStr": "AMD"}),
    ("qd_10_natural", lambda: G.quasi_definite_3d(10, 10, 10, 0.3, 1e-2, seed=4), {"orderingStr": "NATURAL"}),
]


@pytest.mark.parametrize("name,gen,opt", CASES, ids=[c[0] for c in CASES])
def test_ldl_factor_and_solution_match_oracle(name, gen, opt):
    n, cp, ri, v = gen()
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A, **opt)
    f = oracle_for(M, A)
    assert relerr(M.GetFactor(), f.factor()) <= TOL
    rng = np.random.default_rng(5)
    for nrhs in (1, 16, 70):
        b = rng.standard_normal((n, nrhs))
        M.Solve(b)
        x = M.GetSolution(nrhs=nrhs)
        assert relerr(x, f.solve(b)) <= TOL, nrhs
        assert np.linalg.norm(A.matvec(x) - b) / np.linalg.norm(b) < 1e-10


def test_ldl_inertia_of_quasi_definite():
    """Sylvester's law of inertia: D has as many negative entries as the matrix has
    negative vertices (the negative-definite block's size)."""
    n, cp, ri, v = G.quasi_definite_3d(14, 14, 14, 0.35, 1e-2, seed=7)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A)
    neg_vertices = int((v[cp[:-1] - 1] < 0).sum())
    assert int((diag_of_factor(M) < 0).sum()) == neg_vertices


def test_cholesky_rejects_indefinite_and_ldl_accepts_it():
    n, cp, ri, v = G.quasi_definite_3d(10, 10, 10, 0.3, 1e-2, seed=5)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0))
    M.SymbolicFactorization(A)
    M.DistributeMatrix(A)
    with pytest.raises(NotSPDError):
        M.Factorize()
    L = setup(A)
    b = np.random.default_rng(0).standard_normal((n, 2))
    L.Solve(b)
    x = L.GetSolution(nrhs=2)
    assert np.linalg.norm(A.matvec(x) - b) / np.linalg.norm(b) < 1e-12


def test_zero_pivot_is_reported_and_handle_recovers():
    """A zero diagonal entry at the vertex eliminated first: the first pivot is exactly zero."""
    n, cp, ri, v = G.quasi_definite_3d(8, 8, 8, 0.3, 1e-2, seed=6)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0, decomposition="LDL"))
    M.SymbolicFactorization(A)
    perm, _ = M.GetOrdering()
    first = perm[0] - 1  # original vertex of permuted column 0
    bad = v.copy()
    bad[cp[first] - 1] = 0.0  # rows are sorted: a column's first entry is its diagonal
    M.DistributeMatrix(DistSparseMatrix.from_lower_csc(n, cp, ri, bad))
    with pytest.raises(NotSPDError, match="zero pivot"):
        M.Factorize()
    code, sn, col = M.GetStatus()
    assert (code, sn, col) == (1, 0, 0)
    M.DistributeMatrix(A)
    M.Factorize()
    f = oracle_for(M, A)
    assert relerr(M.GetFactor(), f.factor()) <= TOL


def test_ldl_batch_of_mixed_systems():
    """Batched analysis (one forest) with LDL^T: SPD and indefinite systems together."""
    systems = [G.quasi_definite_3d(9, 9, 9, 0.3, 1e-2, seed=1), G.stencil27(10, 10, 10, 1e-2, seed=2),
               G.quasi_definite_3d(7, 11, 5, 0.5, 1e-2, seed=3)]
    n, cp, ri, v, offs = G.block_diagonal(systems)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0, decomposition="LDL"))
    M.SymbolicFactorizationBatch(A, offs)
    M.DistributeMatrix(A)
    M.Factorize()
    b = np.random.default_rng(1).standard_normal((n, 3))
    M.Solve(b)
    x = M.GetSolution(nrhs=3)
    for k, s in enumerate(systems):
        lo, hi = offs[k], offs[k + 1]
        As = DistSparseMatrix.from_lower_csc(*s)
        r = As.matvec(x[lo:hi]) - b[lo:hi]
        assert np.linalg.norm(r) / np.linalg.norm(b[lo:hi]) < 1e-12, k
