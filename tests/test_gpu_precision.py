"""Precision form: FP32 factor (3xTF32 tensor-core updates, FP64 diagonal pivots)
plus FP64 iterative refinement.  Every solution must reach backward error
eta = ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= 1e-12, measured here
against the FP64 matrix, and agree with the FP64 oracle solution to the forward
error that backward error allows (kappa * 1e-12)."""
import os

import numpy as np
import pytest

from oracle import numeric
from sympack_b200 import DistSparseMatrix, SymPACKError, generators as G, symPACKMatrix2D, symPACKOptions

pytestmark = pytest.mark.gpu


def backward_error(A, x, b):
    n = A.size
    r = (b - A.matvec(x)).reshape(n, -1)
    cols = np.repeat(np.arange(n), np.diff(A.colptr))
    rows = A.rowind - 1
    rs = np.zeros(n)
    np.add.at(rs, rows, np.abs(A.nzvalLocal))
    off = rows != cols
    np.add.at(rs, cols[off], np.abs(A.nzvalLocal[off]))
    x2, b2 = x.reshape(n, -1), b.reshape(n, -1)
    return float((np.abs(r).max(0) / (rs.max() * np.abs(x2).max(0) + np.abs(b2).max(0))).max())


def factor(A, precision, **kw):
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0, precision=precision, **kw))
    M.SymbolicFactorization(A)
    M.DistributeMatrix(A)
    M.Factorize()
    return M


@pytest.mark.parametrize("delta,fwd_tol", [(1e-2, 1e-9), (1e-5, 1e-6)])
@pytest.mark.parametrize("k", [12, 18])
def test_fp32_ir_reaches_fp64_backward_error(delta, fwd_tol, k):
    n, cp, ri, v = G.stencil27(k, k, k, delta, seed=2)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = factor(A, "FP32_IR")
    rng = np.random.default_rng(4)
    for nrhs in (1, 16):
        b = rng.standard_normal((n, nrhs))
        M.Solve(b)
        x = M.GetSolution(nrhs=nrhs)
        inf = M.info()
        assert inf.backward_error <= 1e-12
        assert backward_error(A, x, b) <= 1e-12
        # FP64 oracle solution on the same ordering
        perm, invp = M.GetOrdering()
        xl, li = M.GetStructure()
        sym = dict(xsuper=M.GetSupernodalPartition(), xlindx=xl, lindx=li, supmember=M.GetSupMembership(), invp=invp)
        f = numeric.OracleFactor(n, sym, threads=os.cpu_count())
        f.distribute(cp, ri, v)
        f.factorize()
        xo = f.solve(b)
        assert np.max(np.abs(x - xo)) / np.max(np.abs(xo)) <= fwd_tol


@pytest.mark.parametrize("engine", ["tcgen05", "mma.sync", "tcgen05-persistent", "tcgen05-tma"])
@pytest.mark.parametrize("k", [14, 22])
def test_fp32_factor_close_to_fp64_factor(engine, k):
    """FP32 factor (3xTF32 updates on either tensor-core engine) against the FP64
    factor: FP32-level agreement (1e-5 of the largest entry)."""
    n, cp, ri, v = G.stencil27(k, k, k, 1e-2, seed=3)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M32 = factor(A, "FP32_IR", fp32_engine=engine)
    M32.SetProfiling(True)
    M32.DistributeMatrix(A)
    M32.Factorize()
    assert M32.GetProfile()["gemm_dmma"]["launches"] > 0  # 128 x 128 tiles ran
    L32 = M32.GetFactor()
    L64 = factor(A, "FP64").GetFactor()
    assert np.max(np.abs(L32 - L64)) / np.max(np.abs(L64)) <= 1e-5


@pytest.mark.parametrize("k,delta,tol", [(22, 1e-2, 1e-6), (26, 1e-5, 1e-5)])
def test_fp32_persistent_factorization_matches_step_sequence(k, delta, tol):
    """The TMA-fed tcgen05 engine in the persistent factorization (one launch) against the
    same engine in the level-ordered launch sequence: the same tiles and operations in
    another order, so agreement at the level of FP32 rounding in another summation order
    (the updates land by atomic additions, so two factorizations with the same schedule
    already differ: up to 6e-8 of the largest entry at delta 1e-2 and 6e-7 at delta 1e-5,
    where the near-singular pivots amplify it), and refined solutions at backward error
    <= 1e-12 twice in a row (the second factorization reuses the launch with its counters
    cleared)."""
    n, cp, ri, v = G.stencil27(k, k, k, delta, seed=5)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    got = {}
    for sched in ("persistent", "steps"):
        M = factor(A, "FP32_IR", fp32_engine="tcgen05-tma", factor_schedule=sched)
        assert (M.info().factor_launches == 1) == (sched == "persistent")
        got[sched] = M.GetFactor()
        b = np.random.default_rng(7).standard_normal((n, 3))
        for rep in range(2):
            if rep:
                M.DistributeMatrix(A)
                M.Factorize()
            M.Solve(b)
            x = M.GetSolution(nrhs=3)
            assert backward_error(A, x, b) <= 1e-12
        M.close()
    assert np.max(np.abs(got["persistent"] - got["steps"])) / np.max(np.abs(got["steps"])) <= tol


def test_refinement_cap_reports_not_converged():
    n, cp, ri, v = G.stencil27(12, 12, 12, 1e-5, seed=2)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = factor(A, "FP32_IR", ir_max_iter=1, ir_tolerance=1e-16)
    with pytest.raises(SymPACKError) as e:
        M.Solve(np.ones(n))
    assert e.value.code == -8  # SPB_ERR_NOT_CONVERGED


def test_profiling_turned_on_between_refined_solves():
    """Profiling switched on after an unprofiled factorization: the refinement's sweeps
    create their own timing events (regression: they once indexed an empty list)."""
    n, cp, ri, v = G.stencil27(10, 10, 10, 1e-2, seed=5)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = factor(A, "FP32_IR")
    b = np.random.default_rng(3).standard_normal((n, 2))
    M.Solve(b)
    x0 = M.GetSolution(nrhs=2)
    M.SetProfiling(True)
    M.Solve(b)
    x1 = M.GetSolution(nrhs=2)
    M.SetProfiling(False)
    assert backward_error(A, x1, b) <= 1e-12
    assert np.max(np.abs(x1 - x0)) <= 1e-10 * np.max(np.abs(x0))
