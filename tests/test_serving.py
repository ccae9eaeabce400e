"""Serving loop, host side: admission by predicted footprint, LRU eviction with
refactor on a miss, right-hand sides merged against a busy factor, and
overlap of requests.  The numeric handle is replaced by a dense numpy stand-in
so that the dispatcher logic runs without a GPU."""
import threading
import time

import numpy as np
import pytest
import scipy.linalg as sla

from sympack_b200 import generators as G, serving as S
from sympack_b200.solver import DistSparseMatrix


class FakeHandle:
    """Dense stand-in for symPACKMatrix2D: the same calls, numpy arithmetic,
    a short sleep per numeric call so that requests overlap."""
    live_bytes = 0
    peak_bytes = 0
    lock = threading.Lock()
    factorizations = 0

    def __init__(self):
        self.n = 0
        self.bytes = 0

    def Init(self, opt):
        self.opt = opt

    def SymbolicFactorization(self, A):
        self.n = A.size

    def SymbolicFactorizationFrom(self, T):
        self.n = T.n
        self._grow(self.PredictDeviceBytes(nrhs=0))

    def _grow(self, b):
        with FakeHandle.lock:
            FakeHandle.live_bytes += b - self.bytes
            FakeHandle.peak_bytes = max(FakeHandle.peak_bytes, FakeHandle.live_bytes)
        self.bytes = b

    def PredictDeviceBytes(self, precision=None, nrhs=1):
        return 8 * self.n * self.n + 40 * self.n * nrhs

    def DistributeMatrix(self, A):
        D = np.zeros((A.size, A.size))
        cols = np.repeat(np.arange(A.size), np.diff(A.colptr))
        D[A.rowind - 1, cols] = A.nzvalLocal
        self.D = D + np.tril(D, -1).T

    def Factorize(self):
        time.sleep(0.01)
        self.L = np.linalg.cholesky(self.D)
        with FakeHandle.lock:
            FakeHandle.factorizations += 1

    def Solve(self, B):
        time.sleep(0.005)
        B = B.reshape(self.n, -1)
        self._grow(max(self.bytes, self.PredictDeviceBytes(nrhs=B.shape[1])))
        self.X = sla.cho_solve((self.L, True), B)

    def GetSolution(self, nrhs=1):
        return self.X.copy()

    def info(self):
        class I:
            backward_error = 1e-16
            ir_iterations = 0
        return I()

    def close(self):
        self._grow(0)


@pytest.fixture
def fake(monkeypatch):
    monkeypatch.setattr(S, "symPACKMatrix2D", FakeHandle)
    FakeHandle.live_bytes = FakeHandle.peak_bytes = FakeHandle.factorizations = 0
    yield FakeHandle


def lap(k, shift=0.0):
    n, cp, ri, v = G.laplacian_2d(k, k, shift)
    return DistSparseMatrix.from_lower_csc(n, cp, ri, v)


def dense_solve(A, B):
    D = np.zeros((A.size, A.size))
    cols = np.repeat(np.arange(A.size), np.diff(A.colptr))
    D[A.rowind - 1, cols] = A.nzvalLocal
    D = D + np.tril(D, -1).T
    return np.linalg.solve(D, B)


def test_results_match_and_solves_merge(fake):
    rng = np.random.default_rng(0)
    A = lap(8, 0.5)
    svc = S.SolverService(memory_budget=1 << 30, max_inflight=4)
    reqs = [S.Request("factor_solve", "a", rng.standard_normal((A.size, 2)), matrix=A)]
    reqs += [S.Request("solve", "a", rng.standard_normal((A.size, int(rng.integers(1, 4))))) for _ in range(20)]
    futs = [svc.submit(r) for r in reqs]
    res = [f.result(timeout=30) for f in futs]
    svc.close()
    for r, o in zip(reqs, res):
        assert np.allclose(o.x, dense_solve(A, r.rhs), rtol=1e-12, atol=1e-12)
    assert svc.stats["solves"] == 20
    assert svc.stats["solve_batches"] < 20  # solves submitted together ran as merged right-hand sides
    assert max(o.batched for o in res) > 1


def test_admission_respects_budget_and_refactors_after_eviction(fake):
    rng = np.random.default_rng(1)
    mats = {f"m{i}": lap(10 + i, 0.1 * i + 0.1) for i in range(6)}
    one = 8 * 15 * 15 * 15 * 15 + (4 << 20)  # about two factors of these sizes fit
    budget = 2 * one
    svc = S.SolverService(memory_budget=budget, max_inflight=3)
    futs = []
    for fid, A in mats.items():
        futs.append((fid, None, svc.submit(S.Request("factor_solve", fid, rng.standard_normal(A.size), matrix=A))))
    for _, _, f in futs:  # every factorization done: the early factors were evicted to make room
        f.result(timeout=60)
    for fid, A in mats.items():  # solves against evicted factors are refactored on the miss
        b = rng.standard_normal(A.size)
        futs.append((fid, b, svc.submit(S.Request("solve", fid, b))))
    out = [(fid, b, f.result(timeout=60)) for fid, b, f in futs]
    svc.close()
    for fid, b, o in out:
        if b is not None:
            assert np.allclose(o.x, dense_solve(mats[fid], b), rtol=1e-12, atol=1e-12)
    assert svc.stats["evictions"] > 0
    assert svc.stats["refactors"] > 0
    assert FakeHandle.peak_bytes <= budget
    assert FakeHandle.live_bytes == 0


def test_requests_overlap(fake):
    rng = np.random.default_rng(2)
    svc = S.SolverService(memory_budget=1 << 30, max_inflight=4)
    futs = [svc.submit(S.Request("factor_solve", f"f{i}", rng.standard_normal(64), matrix=lap(8, 1.0 + i)))
            for i in range(8)]
    for f in futs:
        f.result(timeout=30)
    svc.close()
    assert svc.stats["max_inflight"] > 1


def test_unknown_factor_is_an_error(fake):
    svc = S.SolverService(memory_budget=1 << 30)
    f = svc.submit(S.Request("solve", "nope", np.zeros(4)))
    with pytest.raises(KeyError):
        f.result(timeout=10)
    svc.close()


def test_stream_is_seeded_and_mixed():
    a = S.request_stream(300, 100.0, seed=3, n_max=20000)
    b = S.request_stream(300, 100.0, seed=3, n_max=20000)
    assert [(t, r.kind, r.factor_id, r.spec[2:]) for t, r in a] == [(t, r.kind, r.factor_id, r.spec[2:]) for t, r in b]
    kinds = [r.kind for _, r in a]
    assert 0.2 < kinds.count("factor_solve") / len(kinds) < 0.4
    assert all(1 <= r.spec[3] <= 64 for _, r in a)
    r = S.materialise(next(r for _, r in a if r.kind == "factor_solve"))
    assert r.matrix.size == r.rhs.shape[0]


def test_cached_solves_are_admitted_before_waiting_factorizations(fake):
    """With factorization slots capped, a solve against a cached factor that arrives after
    several new factorizations does not wait for them."""
    rng = np.random.default_rng(2)
    mats = {f"f{i}": lap(9 + i, 0.2) for i in range(5)}
    A0 = lap(8, 0.5)
    svc = S.SolverService(memory_budget=1 << 30, max_inflight=3, max_factor_inflight=1)
    svc.submit(S.Request("factor_solve", "a", rng.standard_normal(A0.size), matrix=A0)).result(timeout=30)
    order = []
    futs = [svc.submit(S.Request("factor_solve", fid, rng.standard_normal(A.size), matrix=A)) for fid, A in mats.items()]
    b = rng.standard_normal(A0.size)
    fs = svc.submit(S.Request("solve", "a", b))
    for f in futs + [fs]:
        f.add_done_callback(lambda f, order=order: order.append(f))
    assert np.allclose(fs.result(timeout=30).x, dense_solve(A0, b), rtol=1e-12, atol=1e-12)
    [f.result(timeout=60) for f in futs]
    svc.close()
    assert order.index(fs) < len(futs)  # finished before the last factorization
    assert svc.stats["max_inflight"] <= 3


def test_one_slot_serves_cached_solves_and_factorizations(fake):
    """max_inflight=1 (so one factorization slot at most): cached solves and new
    factorizations mixed in one queue all finish; neither class starves the other."""
    rng = np.random.default_rng(4)
    A0 = lap(8, 0.5)
    svc = S.SolverService(memory_budget=1 << 30, max_inflight=1)
    svc.submit(S.Request("factor_solve", "a", rng.standard_normal(A0.size), matrix=A0)).result(timeout=30)
    mats = {f"g{i}": lap(7 + i, 0.3) for i in range(3)}
    futs, checks = [], []
    for i in range(12):
        b = rng.standard_normal(A0.size)
        futs.append(svc.submit(S.Request("solve", "a", b)))
        checks.append((A0, b))
        if i % 4 == 0:
            fid = f"g{i // 4}"
            b2 = rng.standard_normal(mats[fid].size)
            futs.append(svc.submit(S.Request("factor_solve", fid, b2, matrix=mats[fid])))
            checks.append((mats[fid], b2))
    for f, (A, b) in zip(futs, checks):
        assert np.allclose(f.result(timeout=60).x, dense_solve(A, b), rtol=1e-12, atol=1e-12)
    svc.close()
    assert svc.stats["max_inflight"] == 1


def test_oversized_factorization_fails_at_once_and_solves_go_on(fake):
    """A factorization whose predicted footprint exceeds the whole budget is refused
    with MemoryError instead of holding the queue; cached solves keep running."""
    rng = np.random.default_rng(5)
    A0 = lap(6, 0.5)
    big = lap(30, 0.5)  # 8 n^2 bytes = 6.5 MB, above the budget below
    svc = S.SolverService(memory_budget=(4 << 20) + 200_000, max_inflight=2)
    svc.submit(S.Request("factor_solve", "a", rng.standard_normal(A0.size), matrix=A0)).result(timeout=30)
    fb = svc.submit(S.Request("factor_solve", "big", rng.standard_normal(big.size), matrix=big))
    bs = [rng.standard_normal(A0.size) for _ in range(6)]
    fs = [svc.submit(S.Request("solve", "a", b)) for b in bs]
    with pytest.raises(MemoryError):
        fb.result(timeout=30)
    for f, b in zip(fs, bs):
        assert np.allclose(f.result(timeout=30).x, dense_solve(A0, b), rtol=1e-12, atol=1e-12)
    svc.close()
