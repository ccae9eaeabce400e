"""Batching form on the GPU: many uneven systems factored together (every
elimination-tree level of every system in the same launches) give, system by
system, the solution of that system factored alone and of the FP64 oracle."""
import os

import numpy as np
import pytest

from oracle import numeric
from sympack_b200 import DistSparseMatrix, autotune, generators as G, symPACKMatrix2D, symPACKOptions

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def batch_factor(systems, **opt):
    n, cp, ri, v, offs = G.block_diagonal(systems)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0, **opt))
    M.SymbolicFactorizationBatch(A, offs)
    M.DistributeMatrix(A)
    M.Factorize()
    return M, A, offs


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


@pytest.mark.parametrize("nrhs", [1, 8])
def test_batch_fp64_matches_single_and_oracle(nrhs):
    systems = G.batch_systems(24, 60, 4000, seed=7)
    M, A, offs = batch_factor(systems)
    rng = np.random.default_rng(1)
    b = rng.standard_normal((A.size, nrhs))
    M.Solve(b)
    x = M.GetSolution(nrhs=nrhs)
    # oracle on the merged analysis
    perm, invp = M.GetOrdering()
    xl, li = M.GetStructure()
    sym = dict(xsuper=M.GetSupernodalPartition(), xlindx=xl, lindx=li, supmember=M.GetSupMembership(), invp=invp)
    f = numeric.OracleFactor(A.size, sym, threads=os.cpu_count())
    f.distribute(A.colptr, A.rowind, A.nzvalLocal)
    f.factorize()
    xo = f.solve(b)
    for k, s in enumerate(systems[:8]):
        lo, hi = int(offs[k]), int(offs[k + 1])
        assert rel(x[lo:hi], xo[lo:hi]) <= 1e-12
        S = symPACKMatrix2D()
        S.Init(symPACKOptions(device=0))
        As = DistSparseMatrix.from_lower_csc(*s)
        S.SymbolicFactorization(As)
        S.DistributeMatrix(As)
        S.Factorize()
        S.Solve(np.ascontiguousarray(b[lo:hi]))
        assert rel(x[lo:hi], S.GetSolution(nrhs=nrhs)) <= 1e-12
        S.close()
    assert rel(x, xo) <= 1e-12
    M.close()


def test_batch_of_200_named_systems_each_matches_its_own_oracle():
    """200 systems of the batching workload's generator (n log-uniform in [500, 20000],
    Laplacians and random graphs, seed 0) factored as one batch; every system's solution
    is checked against an oracle factorization of that system alone (its own analysis)
    within 1e-12, beside the reference's residual metric (driver/utils.hpp:136-140)."""
    systems = G.batch_systems(200, 500, 20000, seed=0)
    M, A, offs = batch_factor(systems)
    b = np.random.default_rng(4).standard_normal((A.size, 2))
    M.Solve(b)
    x = M.GetSolution(nrhs=2)
    M.close()

    def alone(s):  # host-only analysis of one system by itself (the C calls release the GIL)
        As = DistSparseMatrix.from_lower_csc(*s)
        T = symPACKMatrix2D()
        T.Init(symPACKOptions(device=-1))
        T.SymbolicFactorization(As)
        xl, li = T.GetStructure()
        sym = dict(xsuper=T.GetSupernodalPartition(), xlindx=xl, lindx=li, supmember=T.GetSupMembership(),
                   invp=T.GetOrdering()[1])
        T.close()
        return As, sym

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(os.cpu_count()) as ex:
        analyses = list(ex.map(alone, systems))
    worst = 0.0
    for k, (As, sym) in enumerate(analyses):
        lo, hi = int(offs[k]), int(offs[k + 1])
        f = numeric.OracleFactor(As.size, sym, threads=os.cpu_count())
        f.distribute(As.colptr, As.rowind, As.nzvalLocal)
        f.factorize()
        bk = np.ascontiguousarray(b[lo:hi])
        err = rel(x[lo:hi], f.solve(bk))
        worst = max(worst, err)
        assert err <= 1e-12, (k, As.size, err)
        assert np.linalg.norm(As.matvec(x[lo:hi]) - bk) / np.linalg.norm(bk) < 1e-12, k
    assert worst <= 1e-12


def test_batch_fp32_ir_reaches_backward_error():
    systems = G.batch_systems(20, 60, 3000, seed=11)
    M, A, offs = batch_factor(systems, precision="FP32_IR")
    rng = np.random.default_rng(2)
    b = rng.standard_normal((A.size, 4))
    M.Solve(b)
    x = M.GetSolution(nrhs=4)
    assert M.info().backward_error <= 1e-12
    for k in range(len(systems)):
        lo, hi = int(offs[k]), int(offs[k + 1])
        As = DistSparseMatrix.from_lower_csc(*systems[k])
        assert backward_error(As, x[lo:hi], b[lo:hi]) <= 1e-12
    M.close()


@pytest.mark.parametrize("small_w,big_rows", [(16, 96), (48, 256)])
def test_batch_tile_shapes_do_not_change_result(small_w, big_rows):
    systems = G.batch_systems(10, 200, 3000, seed=5)
    b = np.random.default_rng(3).standard_normal((sum(s[0] for s in systems), 2))
    xs = []
    for opt in (dict(), dict(plan_small_max_w=small_w, plan_big_tile_rows=big_rows)):
        M, A, offs = batch_factor(systems, **opt)
        M.Solve(b)
        xs.append(M.GetSolution(nrhs=2))
        M.close()
    assert rel(xs[1], xs[0]) <= 1e-12


def test_autotune_picks_cached_plan_and_keeps_result(tmp_path, monkeypatch):
    monkeypatch.setenv("SPB_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    systems = G.batch_systems(12, 100, 2500, seed=9)
    n, cp, ri, v, offs = G.block_diagonal(systems)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    b = np.random.default_rng(6).standard_normal(n)
    xs = []
    for expect_cached in (False, True):
        M = symPACKMatrix2D()
        M.Init(symPACKOptions(device=0))
        M.SymbolicFactorizationBatch(A, offs)
        r = autotune.tune(M, A, offs, candidates=[(16, 256), (48, 96)], reps=1)
        assert r["cached"] is expect_cached
        assert (r["small_max_w"], r["big_tile_rows"]) in [(16, 256), (48, 96)]
        M.Factorize()
        M.Solve(b)
        xs.append(M.GetSolution())
        M.close()
    assert (tmp_path / "tune.json").exists()
    assert rel(xs[1], xs[0]) <= 1e-12
