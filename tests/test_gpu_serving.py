"""Serving form on the GPU: each result of the continuous-batching loop is the
same as the request run alone, the footprint used for admission is the
footprint the handle allocates, and a reused symbolic analysis factors exactly
like a fresh one.

Tolerance of "the same": both solutions reach backward error <= 1e-12 against
the FP64 matrix, and they agree to 1e-9 relative (kappa * 1e-12 for the
kappa <= 1e3 matrices of this stream)."""
import numpy as np
import pytest

from sympack_b200 import DistSparseMatrix, generators as G, serving as S, symPACKMatrix2D, symPACKOptions

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


def test_results_same_alone_and_in_the_mix():
    stream = S.request_stream(48, 2000.0, seed=5, n_min=1000, n_max=30000, nrhs_max=8)
    svc = S.SolverService(max_inflight=6, memory_budget=8 << 30)
    S.replay(svc, stream, timeout=300)
    mixed = [r.future.result() for _, r in stream]
    svc.close()
    assert svc.stats["max_inflight"] > 1
    mats = {r.factor_id: r.matrix for _, r in stream if r.kind == "factor_solve"}
    for (_, r), res in zip(stream, mixed):
        A = mats[r.factor_id]
        assert res.backward_error <= 1e-12
        assert backward_error(A, res.x, r.rhs) <= 1e-12
        alone = S.SolverService(max_inflight=1, memory_budget=8 << 30)
        x1 = alone.submit(S.Request("factor_solve", "x", r.rhs, matrix=A)).result(timeout=120).x
        alone.close()
        assert np.abs(res.x - x1).max() <= 1e-9 * np.abs(x1).max()


@pytest.mark.parametrize("precision", ["FP64", "FP32_IR"])
@pytest.mark.parametrize("nrhs", [1, 40])
def test_predicted_footprint_is_allocated_footprint(precision, nrhs):
    n, cp, ri, v = G.stencil27(14, 14, 14, 1e-2)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    T = symPACKMatrix2D()
    T.Init(symPACKOptions(device=-1))
    T.SymbolicFactorization(A)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0, precision=precision))
    M.SymbolicFactorizationFrom(T)
    M.DistributeMatrix(A)
    M.Factorize()
    M.Solve(np.ones((n, nrhs)))
    assert M.info().device_bytes == T.PredictDeviceBytes(precision, nrhs)
    M.close()


def test_reused_analysis_factors_like_a_fresh_one():
    n, cp, ri, v = G.stencil27(16, 16, 16, 1e-2, seed=3)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    T = symPACKMatrix2D()
    T.Init(symPACKOptions(device=-1))
    T.SymbolicFactorization(A)
    out = []
    for reuse in (False, True):
        M = symPACKMatrix2D()
        M.Init(symPACKOptions(device=0))
        if reuse:
            M.SymbolicFactorizationFrom(T)
        else:
            M.SymbolicFactorization(A)
        M.DistributeMatrix(A)
        M.Factorize()
        M.Solve(np.arange(n, dtype=np.float64))
        out.append((M.GetSolution(), M.GetSupernodalPartition(), M.GetOrdering()[0]))
        M.close()
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])
    assert np.abs(out[0][0] - out[1][0]).max() <= 1e-12 * np.abs(out[1][0]).max()
