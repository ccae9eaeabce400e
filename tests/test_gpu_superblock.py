"""Super-block solve: supernodes wider than one 64-column block are solved through
the inverses of their diagonal super-blocks (sb blocks each), computed by the first
solve after a factorization.  Parity with the CPU oracle (substitution) at 1e-12 for
several super-block sizes, roots with a partial last block and super-blocks of one
block, in FP64, LDL^T and FP32 + refinement; refactorization with new values must
recompute the inverses."""
import os

import numpy as np
import pytest

from oracle import numeric
from sympack_b200 import DistSparseMatrix, generators as G, symPACKMatrix2D, symPACKOptions

pytestmark = pytest.mark.gpu
TOL = 1e-12


def factored(A, **opt):
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0, **opt))
    M.SymbolicFactorization(A)
    M.DistributeMatrix(A)
    M.Factorize()
    return M


def oracle_for(M, A, ldl=False):
    perm, invp = M.GetOrdering()
    xl, li = M.GetStructure()
    sym = dict(xsuper=M.GetSupernodalPartition(), xlindx=xl, lindx=li, supmember=M.GetSupMembership(), invp=invp)
    f = numeric.OracleFactor(A.size, sym, threads=os.cpu_count(), ldl=ldl)
    f.distribute(A.colptr, A.rowind, A.nzvalLocal)
    f.factorize()
    return f


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


CASES = [
    ("st27_24", lambda: G.stencil27(24, 24, 24, 1e-2, seed=1)),     # root 1275 columns: 20 blocks, partial last
    ("st27_12_d1e-5", lambda: G.stencil27(12, 12, 12, 1e-5, seed=2)),
    ("lap3d_31x17x9", lambda: G.laplacian_3d(31, 17, 9, 1e-3)),
    ("rand_3000", lambda: G.random_graph_spd(3000, 10, 1.05, seed=9)),  # wide dense supernodes
]


@pytest.mark.parametrize("sb", [1, 3, 8, 32])
@pytest.mark.parametrize("name,gen", CASES, ids=[c[0] for c in CASES])
def test_superblock_solve_matches_oracle(name, gen, sb):
    n, cp, ri, v = gen()
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = factored(A, plan_solve_chunk=sb)
    xs = M.GetSupernodalPartition()
    assert int(np.max(np.diff(xs))) > 64  # some supernode takes the super-block path
    f = oracle_for(M, A)
    rng = np.random.default_rng(7)
    for nrhs in (1, 4, 16, 70):
        b = rng.standard_normal((n, nrhs))
        M.Solve(b)
        assert relerr(M.GetSolution(nrhs=nrhs), f.solve(b)) <= TOL, nrhs
    M.close()


def test_refactorization_recomputes_the_inverses():
    n, cp, ri, v = G.stencil27(16, 16, 16, 1e-2, seed=4)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = factored(A)
    b = np.random.default_rng(3).standard_normal((n, 2))
    M.Solve(b)
    _, _, _, v2 = G.stencil27(16, 16, 16, 1e-2, seed=11)  # same pattern, new values
    A2 = DistSparseMatrix.from_lower_csc(n, cp, ri, v2)
    M.DistributeMatrix(A2)
    M.Factorize()
    M.Solve(b)
    assert relerr(M.GetSolution(nrhs=2), oracle_for(M, A2).solve(b)) <= TOL
    M.close()


def test_superblock_solve_with_refinement():
    n, cp, ri, v = G.stencil27(24, 24, 24, 1e-5, seed=3)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = factored(A, precision="FP32_IR")
    b = np.random.default_rng(1).standard_normal((n, 1))
    M.Solve(b)
    x = M.GetSolution(nrhs=1)
    assert M.info().backward_error <= 1e-12
    # normwise backward error on the host, infinity norms (||A||_inf from the symmetric rows)
    cols = np.repeat(np.arange(n), np.diff(cp))
    rows = ri - 1
    rs = np.zeros(n)
    np.add.at(rs, rows, np.abs(v))
    off = rows != cols
    np.add.at(rs, cols[off], np.abs(v[off]))
    eta = np.abs(A.matvec(x) - b).max() / (rs.max() * np.abs(x).max() + np.abs(b).max())
    assert eta <= 1e-12


@pytest.mark.parametrize("sb", [2, 8])
def test_superblock_solve_with_ldl(sb):
    """LDL^T: the forward sweep uses the inverses of L D's diagonal super-blocks, the
    backward sweep those of the unit L."""
    n, cp, ri, v = G.quasi_definite_3d(20, 20, 20, 0.3, 1e-2, seed=4)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = factored(A, decomposition="LDL", plan_solve_chunk=sb)
    f = oracle_for(M, A, ldl=True)
    b = np.random.default_rng(2).standard_normal((n, 2))
    M.Solve(b)
    assert relerr(M.GetSolution(nrhs=2), f.solve(b)) <= TOL
    M.close()
