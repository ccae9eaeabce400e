"""Allocation-free solve entry point (spb_solve_device_noalloc).

It exists for callers that cannot allocate device memory when they solve — a
service whose device memory is reserved up front and owned by another
allocator, where a cudaMalloc in mid-request could fail, or a latency-critical
caller, for which cudaMalloc may synchronize the device.  Its scratch lives in
a static device array instead of a cudaMalloc'd workspace.  These tests call it
through the C ABI and compare it with spb_solve_device on two calls in a row
(the shared array keeps the previous call's contents), with more than 64
right-hand sides (two passes over the counters) also against the CPU oracle,
and check that oversize requests are refused.  This file is collected last."""
import ctypes as C

import numpy as np
import pytest

from sympack_b200 import DistSparseMatrix, generators as G, symPACKMatrix2D, symPACKOptions
from sympack_b200 import _native as N

pytestmark = pytest.mark.gpu
TOL = 1e-12  # the FP64 parity tolerance used by the other GPU tests


def factored(n, cp, ri, v):
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0))
    M.SymbolicFactorization(A)
    M.DistributeMatrix(A)
    M.Factorize()
    return M


def test_noalloc_solve_matches_solve_device_twice():
    import torch
    n, cp, ri, v = G.stencil27(12, 12, 12, 1e-2, seed=6)
    M = factored(n, cp, ri, v)
    lib = N.load()
    rng = np.random.default_rng(11)
    for nrhs in (16, 3):  # two calls in a row, the second smaller than the first
        B = torch.from_numpy(rng.standard_normal((nrhs, n))).cuda()  # column-major n x nrhs
        X_ref = torch.empty_like(B)
        X_new = torch.full_like(B, float("nan"))
        assert lib.spb_solve_device(M._h, C.c_void_p(B.data_ptr()), C.c_void_p(X_ref.data_ptr()), nrhs, n) == 0
        rc = lib.spb_solve_device_noalloc(M._h, C.c_void_p(B.data_ptr()), C.c_void_p(X_new.data_ptr()), nrhs, n)
        assert rc == 0, lib.spb_last_error(M._h).decode()
        ref, new = X_ref.cpu().numpy(), X_new.cpu().numpy()
        assert np.max(np.abs(new - ref)) <= TOL * np.max(np.abs(ref))


def test_noalloc_solve_beyond_64_columns_matches_solve_device_and_oracle():
    """nrhs = 70 runs the sweeps twice (64 + 6 columns): the counters are cleared
    between the passes and the second pass works on the array past column 64."""
    import torch
    from oracle import numeric
    n, cp, ri, v = G.stencil27(12, 12, 12, 1e-2, seed=7)
    M = factored(n, cp, ri, v)
    lib = N.load()
    rng = np.random.default_rng(12)
    perm, invp = M.GetOrdering()
    xl, li = M.GetStructure()
    sym = dict(xsuper=M.GetSupernodalPartition(), xlindx=xl, lindx=li, supmember=M.GetSupMembership(), invp=invp)
    f = numeric.OracleFactor(n, sym, threads=4)
    f.distribute(cp, ri, v)
    f.factorize()
    for nrhs in (70, 130):  # two calls in a row: 2 and 3 passes
        Bh = rng.standard_normal((n, nrhs))
        B = torch.from_numpy(np.ascontiguousarray(Bh.T)).cuda()  # column-major n x nrhs
        X_ref = torch.empty_like(B)
        X_new = torch.full_like(B, float("nan"))
        assert lib.spb_solve_device(M._h, C.c_void_p(B.data_ptr()), C.c_void_p(X_ref.data_ptr()), nrhs, n) == 0
        rc = lib.spb_solve_device_noalloc(M._h, C.c_void_p(B.data_ptr()), C.c_void_p(X_new.data_ptr()), nrhs, n)
        assert rc == 0, lib.spb_last_error(M._h).decode()
        ref, new = X_ref.cpu().numpy().T, X_new.cpu().numpy().T
        assert np.max(np.abs(new - ref)) <= TOL * np.max(np.abs(ref))
        xo = f.solve(Bh)
        assert np.max(np.abs(new - xo)) <= TOL * np.max(np.abs(xo))


def test_noalloc_rejects_requests_beyond_its_scratch():
    import torch
    n, cp, ri, v = G.laplacian_2d(40, 40)
    M = factored(n, cp, ri, v)
    lib = N.load()
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    too_many = (4 * 1024 * 1024) // n + 1  # n * nrhs just above the 4 Mi entries of the array
    rc = lib.spb_solve_device_noalloc(M._h, C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()),
                                      too_many, n)
    assert rc == N.SPB_ERR_INVALID
    assert "exceeds" in lib.spb_last_error(M._h).decode()


def test_noalloc_solve_with_ldl_factor():
    """LDL^T handles solve forward with L D and backward with unit L, here too."""
    import torch
    n, cp, ri, v = G.quasi_definite_3d(12, 12, 12, 0.3, 1e-2, seed=8)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=0, decomposition="LDL"))
    M.SymbolicFactorization(A)
    M.DistributeMatrix(A)
    M.Factorize()
    lib = N.load()
    B = torch.from_numpy(np.random.default_rng(2).standard_normal((4, n))).cuda()
    X_ref, X = torch.empty_like(B), torch.full_like(B, float("nan"))
    assert lib.spb_solve_device(M._h, C.c_void_p(B.data_ptr()), C.c_void_p(X_ref.data_ptr()), 4, n) == 0
    rc = lib.spb_solve_device_noalloc(M._h, C.c_void_p(B.data_ptr()), C.c_void_p(X.data_ptr()), 4, n)
    assert rc == 0, lib.spb_last_error(M._h).decode()
    ref, new = X_ref.cpu().numpy(), X.cpu().numpy()
    assert np.max(np.abs(new - ref)) <= TOL * np.max(np.abs(ref))
