"""GPU factor / solve parity with the CPU oracle (restatement of the reference's
2D cell algorithm), all through the C ABI.  Tolerance: 1e-12 relative (max-norm)
for both the factor and the solution, the north-star bound for the FP64 path."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import numeric
from sympack_b200 import (DeviceTimeoutError, DistSparseMatrix, NotSPDError, StateError, generators as G,
                          symPACKMatrix2D, symPACKOptions)
from sympack_b200 import _native as N

pytestmark = pytest.mark.gpu
TOL = 1e-12


def setup(A, **opt):
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0, **opt))
    M.SymbolicFactorization(A)
    M.DistributeMatrix(A)
    M.Factorize()
    return M


def oracle_for(M, A):
    perm, invp = M.GetOrdering()
    xl, li = M.GetStructure()
    sym = dict(xsuper=M.GetSupernodalPartition(), xlindx=xl, lindx=li, supmember=M.GetSupMembership(), invp=invp)
    f = numeric.OracleFactor(A.size, sym, threads=os.cpu_count())
    f.distribute(A.colptr, A.rowind, A.nzvalLocal)
    f.factorize()
    return f


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


CASES = [
    ("lap3d_20", lambda: G.laplacian_3d(20, 20, 20, 1e-3)),
    ("st27_14", lambda: G.stencil27(14, 14, 14, 1e-2, seed=1)),
    ("st27_12_d1e-5", lambda: G.stencil27(12, 12, 12, 1e-5, seed=2)),
    ("lap3d_31x17x9", lambda: G.laplacian_3d(31, 17, 9, 1e-3)),
    ("rand_3000", lambda: G.random_graph_spd(3000, 10, 1.05, seed=9)),
    ("rand_500_forest", lambda: G.random_graph_spd(500, 1.2, 1.05, seed=5)),
]


@pytest.mark.parametrize("name,gen", CASES)
def test_factor_and_solution_match_oracle(name, gen):
    n, cp, ri, v = gen()
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A)
    f = oracle_for(M, A)
    assert relerr(M.GetFactor(), f.factor()) <= TOL
    rng = np.random.default_rng(3)
    for nrhs in (1, 16, 70):
        b = rng.standard_normal((n, nrhs))
        M.Solve(b)
        x = M.GetSolution(nrhs=nrhs)
        assert relerr(x, f.solve(b)) <= TOL, nrhs


@pytest.mark.parametrize("name,gen", [CASES[0], CASES[4], CASES[5]])
@pytest.mark.parametrize("ordering", ["AMD", "RCM", "NATURAL"])
def test_other_orderings_match_oracle(name, gen, ordering):
    """AMD, RCM and NATURAL orderings (RCM and NATURAL give long chains of
    supernodes: deep elimination trees, few per level): the same bound as MMD."""
    n, cp, ri, v = gen()
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A, orderingStr=ordering)
    f = oracle_for(M, A)
    assert relerr(M.GetFactor(), f.factor()) <= TOL
    b = np.random.default_rng(4).standard_normal((n, 3))
    M.Solve(b)
    assert relerr(M.GetSolution(nrhs=3), f.solve(b)) <= TOL


def test_cfg1_through_rutherford_boeing(tmp_path):
    """2D 5-point Laplacian 64x64 written to RB and read back, as the reference driver does."""
    n, cp, ri, v = G.laplacian_2d(64, 64)
    p = str(tmp_path / "lap2d_64.rb")
    DistSparseMatrix.from_lower_csc(n, cp, ri, v).write_rb(p)
    A = DistSparseMatrix.from_rb(p)
    M = setup(A)
    f = oracle_for(M, A)
    assert relerr(M.GetFactor(), f.factor()) <= TOL
    b = np.random.default_rng(0).uniform(-1.0, 1.0, size=(n, 1))
    M.Solve(b)
    x = M.GetSolution(nrhs=1)
    assert relerr(x, f.solve(b)) <= TOL
    # reference residual metric ||AX - B||_F / ||B||_F (driver/utils.hpp:136-140)
    assert np.linalg.norm(A.matvec(x) - b) / np.linalg.norm(b) < 1e-13


def test_full_size_cfg2_solution_matches_oracle():
    n, cp, ri, v = G.laplacian_3d(60, 60, 60, 1e-3)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A)
    f = oracle_for(M, A)
    b = np.random.default_rng(0).standard_normal((n, 16))
    M.Solve(b)
    x = M.GetSolution(nrhs=16)
    assert relerr(x, f.solve(b)) <= TOL
    assert np.linalg.norm(A.matvec(x) - b) / np.linalg.norm(b) < 1e-14


def chunked_relerr(a, b, chunk=1 << 26):
    """max|a - b| / max|b| without a full-size temporary (the 80^3 factor is 10.8 GB)."""
    num = den = 0.0
    for i in range(0, len(b), chunk):
        num = max(num, float(np.max(np.abs(a[i:i + chunk] - b[i:i + chunk]))))
        den = max(den, float(np.max(np.abs(b[i:i + chunk]))))
    return num / den


def test_full_size_cfg3_fp64_factor_and_solution_match_oracle():
    """Precision-form matrix (27-point stencil 80^3, delta 1e-2, seed 0; n = 512,000,
    1.36e9 factor entries) factored by the plain FP64 path: factor and solution within
    1e-12 of the oracle, and the reference's residual metric (driver/utils.hpp:136-140)."""
    n, cp, ri, v = G.stencil27(80, 80, 80, 1e-2, seed=0)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A)
    f = oracle_for(M, A)
    Lg = M.GetFactor()
    Lo = f.factor()
    ferr = chunked_relerr(Lg, Lo)
    del Lg, Lo
    assert ferr <= TOL
    b = np.random.default_rng(0).standard_normal((n, 2))
    M.Solve(b)
    x = M.GetSolution(nrhs=2)
    M.close()
    assert relerr(x, f.solve(b)) <= TOL
    assert np.linalg.norm(A.matvec(x) - b) / np.linalg.norm(b) < 1e-13


def test_device_solve_with_leading_dimension():
    import torch
    n, cp, ri, v = G.stencil27(9, 9, 9, 1e-2)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A)
    ld = n + 7
    B = np.zeros((3, ld))
    B[:, :n] = np.random.default_rng(1).standard_normal((3, n))
    dB = torch.from_numpy(B).cuda()
    dX = torch.full_like(dB, 7.0)
    M.SolveDevice(dB.data_ptr(), dX.data_ptr(), 3, ld)
    X = dX.cpu().numpy()
    assert np.all(X[:, n:] == 7.0)  # padding untouched
    M.Solve(B[:, :n].T.copy())
    # scatter-adds use atomics: summation order, hence the last bits, may differ run to run
    assert relerr(X[:, :n].T, M.GetSolution(nrhs=3)) <= 1e-14


def test_refactorization_with_new_values_reuses_structure():
    n, cp, ri, v = G.stencil27(11, 11, 11, 1e-2, seed=4)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A)
    _, cp2, ri2, v2 = G.stencil27(11, 11, 11, 1e-2, seed=7)  # same pattern, new values
    assert np.array_equal(cp2, cp) and np.array_equal(ri2, ri)
    A2 = DistSparseMatrix.from_lower_csc(n, cp, ri, v2)
    with pytest.raises(StateError):
        M.Factorize()  # already factored: distribute first
    M.DistributeMatrix(A2)
    M.Factorize()
    f = oracle_for(M, A2)
    assert relerr(M.GetFactor(), f.factor()) <= TOL


def test_not_spd_is_reported_and_handle_recovers():
    n, cp, ri, v = G.laplacian_3d(12, 12, 12, 1e-3)
    bad = v.copy()
    bad[cp[700] - 1] = -1.0  # diagonal entry of column 701
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    Abad = DistSparseMatrix.from_lower_csc(n, cp, ri, bad)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0))
    M.SymbolicFactorization(A)
    M.DistributeMatrix(Abad)
    with pytest.raises(NotSPDError):
        M.Factorize()
    code, sn, col = M.GetStatus()
    assert code == 1 and sn >= 0 and col >= 0
    M.DistributeMatrix(A)
    M.Factorize()
    assert M.GetStatus()[0] == 0
    f = oracle_for(M, A)
    assert relerr(M.GetFactor(), f.factor()) <= TOL


def test_calls_out_of_order_on_device():
    n, cp, ri, v = G.laplacian_2d(10, 10)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0))
    M.SymbolicFactorization(A)
    with pytest.raises(StateError):
        M.Factorize()
    M.DistributeMatrix(A)
    with pytest.raises(StateError):
        M.Solve(np.ones(n))
    M.Factorize()
    with pytest.raises(StateError):
        M.GetSolution(nrhs=1)


def test_profiled_run_matches_graph_run():
    n, cp, ri, v = G.stencil27(13, 13, 13, 1e-2, seed=3)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A)
    L1 = M.GetFactor()
    M.SetProfiling(True)
    M.DistributeMatrix(A)
    M.Factorize()
    L2 = M.GetFactor()
    prof = M.GetProfile()
    assert relerr(L2, L1) <= TOL
    assert sum(p["launches"] for k, p in prof.items() if k not in ("solve_forward", "solve_backward")) >= 1
    assert all(p["ms"] >= 0 for p in prof.values())


TIMEOUT_CHILD = r"""
import sys
sys.path.insert(0, sys.argv[1])
import numpy as np
from sympack_b200 import DeviceTimeoutError, DistSparseMatrix, generators as G, symPACKMatrix2D, symPACKOptions
n, cp, ri, v = G.laplacian_3d(10, 10, 10, 1e-3)
A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
M = symPACKMatrix2D()
M.Init(symPACKOptions(device=0))
M.SymbolicFactorization(A)
M.DistributeMatrix(A)
M.Factorize()
b = np.random.default_rng(0).standard_normal((n, 1))
M.Solve(b)
x_ok = M.GetSolution(nrhs=1)
M.SetWaitLimit(2000)
M.DebugStall(M.info().nsuper - 1)
try:
    M.Solve(b)
    print("NO_TIMEOUT")
    sys.exit(1)
except DeviceTimeoutError:
    pass
M.DebugStall(-1)
M.SetWaitLimit(1 << 24)
M.Solve(b)
err = np.max(np.abs(M.GetSolution(nrhs=1) - x_ok)) / np.max(np.abs(x_ok))
print("RECOVERED", err)
sys.exit(0 if err <= 1e-14 else 2)
"""


def test_solve_wait_timeout_is_reported_and_recovers():
    """A forward wait on an update nobody sends runs out (bounded device wait);
    the call reports a timeout and the next solve on the same handle succeeds.
    Runs in a child process with its own time limit."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", TIMEOUT_CHILD, root], capture_output=True, text=True, timeout=180)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "RECOVERED" in r.stdout


FACTOR_TIMEOUT_CHILD = r"""
import sys
sys.path.insert(0, sys.argv[1])
import numpy as np
from sympack_b200 import DeviceTimeoutError, DistSparseMatrix, generators as G, symPACKMatrix2D, symPACKOptions
n, cp, ri, v = G.laplacian_3d(12, 12, 12, 1e-3)
A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
M = symPACKMatrix2D()
M.Init(symPACKOptions(device=0))
M.SymbolicFactorization(A)
M.DistributeMatrix(A)
M.Factorize()
b = np.random.default_rng(0).standard_normal((n, 1))
M.Solve(b)
x_ok = M.GetSolution(nrhs=1)
M.SetWaitLimit(2000)
M.DebugStallFactor(M.info().nsuper - 1)  # the root waits for one external update too many
M.DistributeMatrix(A)
try:
    M.Factorize()
    print("NO_TIMEOUT")
    sys.exit(1)
except DeviceTimeoutError:
    pass
M.DebugStallFactor(-1)
M.SetWaitLimit(1 << 24)
M.DistributeMatrix(A)
M.Factorize()
M.Solve(b)
err = np.max(np.abs(M.GetSolution(nrhs=1) - x_ok)) / np.max(np.abs(x_ok))
print("RECOVERED", err)
sys.exit(0 if err <= 1e-14 else 2)
"""


def test_factor_wait_timeout_is_reported_and_recovers():
    """The persistent factorization's bounded waits: a supernode waits for an external
    update nobody sends, the call reports a timeout, and the same handle factors again
    afterwards.  Runs in a child process with its own time limit."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", FACTOR_TIMEOUT_CHILD, root], capture_output=True, text=True, timeout=180)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "RECOVERED" in r.stdout


@pytest.mark.parametrize("schedule", ["persistent", "steps"])
def test_factor_schedules_match_oracle(schedule):
    """The persistent factorization and the level-ordered launch sequence give the
    oracle's factor within the parity bound (FP64 Cholesky and LDL^T)."""
    for name, gen, dec in (("st27_16", lambda: G.stencil27(16, 16, 16, 1e-2, seed=8), "LL"),
                           ("rand_3000", lambda: G.random_graph_spd(3000, 10, 1.05, seed=9), "LL"),
                           ("qd_14", lambda: G.quasi_definite_3d(14, 14, 14, 0.3, 1e-2, seed=3), "LDL")):
        n, cp, ri, v = gen()
        A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
        M = setup(A, factor_schedule=schedule, decomposition=dec)
        perm, invp = M.GetOrdering()
        xl, li = M.GetStructure()
        sym = dict(xsuper=M.GetSupernodalPartition(), xlindx=xl, lindx=li, supmember=M.GetSupMembership(), invp=invp)
        f = numeric.OracleFactor(A.size, sym, threads=os.cpu_count(), ldl=dec == "LDL")
        f.distribute(A.colptr, A.rowind, A.nzvalLocal)
        f.factorize()
        assert relerr(M.GetFactor(), f.factor()) <= TOL, name
        assert M.info().factor_launches == (1 if schedule == "persistent" else M.info().factor_launches)
        M.close()


def test_solve_trace_of_a_profiled_solve():
    n, cp, ri, v = G.laplacian_3d(14, 14, 14, 1e-3)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0))
    M.SymbolicFactorization(A)
    M.DistributeMatrix(A)
    M.Factorize()
    M.SetProfiling(True)
    M.Solve(np.ones(n))
    # 4: a small supernode in one task, 6: a batch of tiny leaves (one per thread)
    for sweep, kinds in ((0, {0, 1, 2, 4, 5, 6}), (1, {0, 1, 3, 4, 5, 6})):
        tr = M.GetSolveTrace(sweep).astype(np.int64)
        assert tr.shape[1] == 4 and len(tr) > 0
        t0, t1, t2, sk = tr.T
        assert np.all(t0 > 0) and np.all(t1 >= t0) and np.all(t2 >= t1)
        assert set(np.unique(sk & 255)) <= kinds
        assert np.all((sk >> 8) < M.info().nsuper)
    M.close()


@pytest.mark.parametrize("opt", [dict(plan_outer_nb=64), dict(plan_outer_nb=512), dict(plan_solve_chunk=1),
                                 dict(plan_solve_chunk=3), dict(plan_small_max_w=16, plan_big_tile_rows=96),
                                 dict(plan_small_max_w=48, plan_big_tile_rows=256)],
                         ids=["outer64", "outer512", "superblock1", "superblock3", "small16_rows96", "small48_rows256"])
def test_plan_options_give_the_same_factor_and_solution(opt):
    """Every plan tunable changes only the schedule: factor and solution stay within the
    parity bound of the oracle."""
    n, cp, ri, v = G.stencil27(16, 16, 16, 1e-2, seed=8)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A, **opt)
    f = oracle_for(M, A)
    assert relerr(M.GetFactor(), f.factor()) <= TOL
    b = np.random.default_rng(6).standard_normal((n, 5))
    M.Solve(b)
    assert relerr(M.GetSolution(nrhs=5), f.solve(b)) <= TOL


@pytest.mark.parametrize("decomposition", ["LL", "LDL"])
@pytest.mark.parametrize("case", ["n1", "diag7", "path2", "isolated"])
def test_degenerate_matrices(case, decomposition):
    """One unknown, a diagonal matrix, a single edge, and a path with an isolated vertex:
    one-column supernodes through the small-panel kernel and the fused solve tasks."""
    if case == "n1":
        n, cp, ri, v = 1, np.array([1, 2], np.int64), np.array([1], np.int32), np.array([4.0])
    elif case == "diag7":
        n, cp, ri, v = 7, np.arange(1, 9, dtype=np.int64), np.arange(1, 8, dtype=np.int32), np.arange(1.0, 8.0)
    elif case == "path2":
        n, cp, ri, v = 2, np.array([1, 3, 4], np.int64), np.array([1, 2, 2], np.int32), np.array([3.0, -1.0, 2.0])
    else:  # vertices 1-2-3 on a path, vertex 4 alone
        n = 4
        cp = np.array([1, 3, 5, 6, 7], np.int64)
        ri = np.array([1, 2, 2, 3, 3, 4], np.int32)
        v = np.array([4.0, -1.0, 4.0, -1.0, 4.0, 2.5])
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A, decomposition=decomposition)
    D = np.zeros((n, n))
    cols = np.repeat(np.arange(n), np.diff(cp))
    D[ri - 1, cols] = v
    D = D + np.tril(D, -1).T
    b = np.random.default_rng(0).standard_normal((n, 2))
    M.Solve(b)
    x = M.GetSolution(nrhs=2)
    assert relerr(x, np.linalg.solve(D, b)) <= TOL


def test_dump_matlab_of_the_device_factor_matches_the_oracle(tmp_path):
    """symPACKMatrix2D::DumpMatlab (2D.hpp:6762-6854): the device factor as MATLAB text,
    read back, equals the oracle's factor in the same form."""
    import io
    from sympack_b200.solver import matlab_sparse
    n, cp, ri, v = G.laplacian_3d(9, 8, 7, 1e-2)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A)
    buf = io.StringIO()
    M.DumpMatlab(buf)
    path = tmp_path / "L.m"
    M.DumpMatlab(str(path))
    assert path.read_text() == buf.getvalue()
    f = oracle_for(M, A)
    xl, li = M.GetStructure()
    ref = matlab_sparse(n, M.GetSupernodalPartition(), xl, li, f.factor())

    def parse(text):
        head, tail = text.split("],[", 2)[:2], text.split("],[", 2)[2]
        rows = np.array(head[0][len("+sparse(["):].split(), np.int64)
        cols = np.array(head[1].split(), np.int64)
        vals = np.array(tail.split("]")[0].split(), np.float64)
        return rows, cols, vals

    rg, cg, vg = parse(buf.getvalue())
    ro, co, vo = parse(ref)
    np.testing.assert_array_equal(rg, ro)
    np.testing.assert_array_equal(cg, co)
    assert relerr(vg, vo) <= TOL
    assert buf.getvalue().endswith(f"],{n},{n})\n")
    M.close()


def test_profile_guided_task_order_keeps_the_factor():
    """spb_reorder_factor_from_trace: the persistent factorization re-ordered by the
    measured task durations of a traced run gives the same factor (within the FP64
    tolerance: the atomic update order may differ) and matches the oracle."""
    n, cp, ri, v = G.laplacian_3d(20, 20, 20, 1e-3)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = setup(A)
    L0 = M.GetFactor()
    with pytest.raises(StateError):
        M.ReorderFactorFromTrace()  # no traced factorization yet
    pred = M.TuneFactorOrder(A, passes=2)
    assert len(pred) == 2 and all(p > 0 for p in pred)
    with pytest.raises(StateError):
        M.ReorderFactorFromTrace()  # the trace is used up
    M.Factorize()
    L1 = M.GetFactor()
    assert relerr(L1, L0) <= TOL
    f = oracle_for(M, A)
    assert relerr(L1, f.factor()) <= TOL
    M.close()
