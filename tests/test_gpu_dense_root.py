"""Dense-root solve in one thread-block cluster (solves of at most 4 right-hand sides on
a root supernode with no off-diagonal rows): parity with the CPU oracle at 1e-12 and
agreement with the persistent sweep (dense path disabled), in FP64, FP32 + refinement
and LDL^T.  The threshold is lowered so that small matrices take the path; the root
widths cover fewer blocks than cluster CTAs (ranks without blocks) and many blocks
with a partial last block."""
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


def root_width(M):
    xs = M.GetSupernodalPartition()
    return int(xs[-1] - xs[-2])


CASES = [
    ("st27_24", lambda: G.stencil27(24, 24, 24, 1e-2, seed=1), 256),     # root 1275: 20 blocks, partial last
    ("st27_12", lambda: G.stencil27(12, 12, 12, 1e-2, seed=2), 64),      # a few blocks, idle ranks
    ("lap3d_31x17x9", lambda: G.laplacian_3d(31, 17, 9, 1e-3), 64),
]


@pytest.mark.parametrize("name,gen,minw", CASES, ids=[c[0] for c in CASES])
def test_dense_root_solve_matches_oracle_and_persistent_sweep(name, gen, minw):
    n, cp, ri, v = gen()
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = factored(A, plan_dense_min_w=minw)
    Mp = factored(A, plan_dense_min_w=-1)
    assert root_width(M) >= minw
    f = oracle_for(M, A)
    rng = np.random.default_rng(7)
    for nrhs in (1, 3, 4, 5):  # 5 takes the persistent path for the root too
        b = rng.standard_normal((n, nrhs))
        M.Solve(b)
        x = M.GetSolution(nrhs=nrhs)
        assert relerr(x, f.solve(b)) <= TOL, nrhs
        Mp.Solve(b)
        assert relerr(x, Mp.GetSolution(nrhs=nrhs)) <= 1e-13, nrhs


def test_dense_root_with_refinement():
    n, cp, ri, v = G.stencil27(24, 24, 24, 1e-5, seed=3)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = factored(A, precision="FP32_IR", plan_dense_min_w=256)
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


def test_dense_root_with_ldl():
    n, cp, ri, v = G.quasi_definite_3d(20, 20, 20, 0.3, 1e-2, seed=4)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = factored(A, decomposition="LDL", plan_dense_min_w=128)
    f = oracle_for(M, A, ldl=True)
    b = np.random.default_rng(2).standard_normal((n, 2))
    M.Solve(b)
    assert relerr(M.GetSolution(nrhs=2), f.solve(b)) <= TOL
