"""Serving form: a continuous-batching request loop over device-cached factors.

Two request kinds arrive over time:

* ``factor_solve`` — a fresh SPD matrix plus right-hand sides; the factor is
  kept on the device under ``factor_id`` afterwards;
* ``solve`` — right-hand sides against a factor cached earlier.

The loop (one dispatcher thread) admits requests as execution slots and HBM
free up, so requests that arrive while others run start at once and their work
overlaps on the device (every factor lives in its own handle with its own CUDA
stream; the numeric calls release the GIL).  Admission of a factorization is by
the device footprint predicted from its symbolic factor
(``PredictDeviceBytes``) against a memory budget; idle cached factors are
evicted least-recently-used to make room, keeping the host matrix (of the
latest ``max_evicted_kept`` evictions) so that a later solve against an evicted
factor refactors it.  Solve requests waiting on
the same cached factor are merged into one multi-right-hand-side solve (up to
``max_batch_rhs`` columns), which is what a triangular solve is fastest at.
Symbolic analyses are cached by sparsity pattern, so a fresh matrix on a known
pattern skips the host ordering (``SymbolicFactorizationFrom``); analyses of
new patterns run on a separate host thread pool and never hold a GPU slot.

Results are the same as a request run alone: the numeric path of a request
does not depend on what else is running (separate handles, separate buffers),
and with FP32 + iterative refinement every result meets the backward-error
target by itself.
"""
from __future__ import annotations

import collections
import hashlib
import threading
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from .solver import DistSparseMatrix, symPACKMatrix2D, symPACKOptions

ALLOC_SLACK = 4 << 20  # per handle: device allocator granularity, stream, events


@dataclass(eq=False)
class Request:
    kind: str                          # "factor_solve" | "solve"
    factor_id: str
    rhs: np.ndarray | None             # n or n x nrhs, float64, original ordering
    matrix: DistSparseMatrix | None = None
    spec: tuple | None = None          # stream request not yet materialised: (pattern, seed, n, nrhs)
    keep: bool = True                  # keep the solution in the result (False: backward error etc. only)
    t_submit: float = 0.0
    t_start: float = 0.0
    t_done: float = 0.0
    batched: int = 1                   # requests in the solve this one ran in
    refactored: bool = False           # solve against an evicted factor: factored again
    need: int = 0                      # predicted device bytes of its factorization (0 = not yet known)
    future: Future = field(default_factory=Future, repr=False)

    @property
    def nrhs(self) -> int:
        return 1 if self.rhs.ndim == 1 else int(self.rhs.shape[1])

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


@dataclass
class Result:
    x: np.ndarray
    backward_error: float
    ir_iterations: int
    latency_s: float
    queue_s: float
    batched: int
    refactored: bool


class _Factor:
    __slots__ = ("M", "bytes", "busy", "matrix", "key", "n")

    def __init__(self, M, nbytes, matrix, key, n):
        self.M, self.bytes, self.busy, self.matrix, self.key, self.n = M, nbytes, True, matrix, key, n


class SolverService:
    """Continuous-batching factor / solve service on one GPU."""

    def __init__(self, device: int = 0, precision: str = "FP32_IR", max_inflight: int = 8,
                 memory_budget: int | None = None, max_batch_rhs: int = 64, ir_tolerance: float = 1e-12,
                 analysis_threads: int = 4, max_evicted_kept: int = 64, max_factor_inflight: int | None = None):
        self.device, self.precision = device, precision
        self.max_inflight, self.max_batch_rhs, self.ir_tolerance = max_inflight, max_batch_rhs, ir_tolerance
        # factorizations may hold at most this many slots, so that solves against cached
        # factors (short) always find one
        self.max_factor_inflight = max(1, max_inflight - 2 if max_factor_inflight is None else max_factor_inflight)
        self._factor_inflight = 0
        if memory_budget is None:
            import torch  # device memory query only
            free, _ = torch.cuda.mem_get_info(device)
            memory_budget = int(free * 0.7)
        self.memory_budget = int(memory_budget)
        self.max_evicted_kept = max_evicted_kept
        self._cv = threading.Condition()
        self._waiting: collections.deque[Request] = collections.deque()
        self._factors: collections.OrderedDict[str, _Factor] = collections.OrderedDict()  # LRU order
        self._evicted: dict[str, tuple] = {}     # factor_id -> (matrix, pattern key)
        self._pending_ids: set[str] = set()      # factor ids being factored
        self._patterns: dict[str, Future] = {}   # pattern key -> Future[host-only analysed handle]
        self._pattern_memo: dict[int, tuple] = {}
        self._reserved = 0
        self._inflight = 0
        self._stop = False
        self.stats = collections.Counter()
        self.done: list[Request] = []
        self._workers = ThreadPoolExecutor(max_inflight, thread_name_prefix="spb-serve")
        self._analysis = ThreadPoolExecutor(analysis_threads, thread_name_prefix="spb-analyse")
        self._thread = threading.Thread(target=self._loop, name="spb-dispatch", daemon=True)
        self._thread.start()

    # -- public -----------------------------------------------------------------
    def submit(self, req: Request) -> Future:
        req.t_submit = time.perf_counter()
        if req.rhs.dtype != np.float64:
            req.rhs = req.rhs.astype(np.float64)
        if req.kind == "factor_solve":
            if req.matrix is None:
                raise ValueError("factor_solve needs a matrix")
            self._ensure_pattern(req.matrix)
        elif req.kind != "solve":
            raise ValueError(f"unknown request kind {req.kind!r}")
        with self._cv:
            self._waiting.append(req)
            self._cv.notify_all()
        return req.future

    def drain(self, timeout: float | None = None) -> None:
        """Wait until every submitted request has finished."""
        end = None if timeout is None else time.perf_counter() + timeout
        with self._cv:
            while self._waiting or self._inflight:
                left = None if end is None else end - time.perf_counter()
                if left is not None and left <= 0:
                    raise TimeoutError("serving queue did not drain")
                self._cv.wait(timeout=0.05 if left is None else min(left, 0.05))

    def close(self) -> None:
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        self._thread.join()
        self._workers.shutdown(wait=True)
        self._analysis.shutdown(wait=True)
        for F in self._factors.values():
            F.M.close()
        self._factors.clear()
        for fut in self._patterns.values():
            if fut.done() and fut.exception() is None:
                fut.result().close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def cached_bytes(self) -> int:
        with self._cv:
            return sum(F.bytes for F in self._factors.values())

    # -- symbolic analyses by pattern ---------------------------------------------
    def _pattern_key(self, A: DistSparseMatrix) -> str:
        memo = self._pattern_memo.get(id(A.rowind))
        if memo is not None and memo[0] is A.rowind and memo[1] is A.colptr:
            return memo[2]
        h = hashlib.blake2b(digest_size=16)
        h.update(np.ascontiguousarray(A.colptr, np.int64).tobytes())
        h.update(np.ascontiguousarray(A.rowind, np.int32).tobytes())
        key = h.hexdigest()
        self._pattern_memo[id(A.rowind)] = (A.rowind, A.colptr, key)
        return key

    def _ensure_pattern(self, A: DistSparseMatrix) -> str:
        key = self._pattern_key(A)
        with self._cv:
            if key not in self._patterns:
                self._patterns[key] = self._analysis.submit(self._analyse, A)
                self._patterns[key].add_done_callback(lambda _f: self._notify())
        return key

    def _analyse(self, A: DistSparseMatrix) -> symPACKMatrix2D:
        # analysed with the service's precision: its plan is the one the factor handles use
        T = symPACKMatrix2D()
        T.Init(symPACKOptions(device=-1, precision=self.precision))
        T.SymbolicFactorization(A)
        return T

    def _notify(self):
        with self._cv:
            self._cv.notify_all()

    # -- dispatcher -----------------------------------------------------------------
    def _loop(self):
        while True:
            with self._cv:
                if self._stop and not self._waiting and not self._inflight:
                    return
                try:
                    jobs = self._admit()
                except BaseException as e:  # noqa: BLE001 - a dispatcher bug fails the queue instead of hanging it
                    for r in self._waiting:
                        if not r.future.done():
                            r.future.set_exception(e)
                    self._waiting.clear()
                    self._cv.notify_all()
                    continue
                if not jobs:
                    self._cv.wait(timeout=0.05)
                    continue
            for job in jobs:
                self._workers.submit(self._run, job)

    def _evict(self, need: int) -> bool:
        """Free idle cached factors (LRU first) until need more bytes fit."""
        waited_on = {r.factor_id for r in self._waiting if r.kind == "solve"}
        for pass_ in (0, 1):  # first factors nobody waits on, then any idle one
            for fid in list(self._factors):
                if self._reserved + need <= self.memory_budget:
                    return True
                F = self._factors[fid]
                if F.busy or (pass_ == 0 and fid in waited_on):
                    continue
                del self._factors[fid]
                self._evicted[fid] = (F.matrix, F.key)
                while len(self._evicted) > self.max_evicted_kept:  # oldest evictions are forgotten
                    self._evicted.pop(next(iter(self._evicted)))
                self._reserved -= F.bytes
                F.M.close()
                self.stats["evictions"] += 1
        return self._reserved + need <= self.memory_budget

    def _admit(self) -> list:
        """Start what fits: first the solves whose factor is cached (short jobs, right-hand
        sides merged per factor; they leave one slot free while a factorization that could
        start now waits),
        then factorizations, each class in arrival order; factorizations are capped at
        max_factor_inflight slots."""
        jobs = []
        self._admit_pass(jobs, solves=True)
        self._admit_pass(jobs, solves=False)
        self._inflight += len(jobs)
        self._factor_inflight += sum(1 for j in jobs if j[0] == "factor")
        self.stats["max_inflight"] = max(self.stats["max_inflight"], self._inflight)
        return jobs

    def _factor_need(self, req: Request):
        """(matrix, pattern key, analysed handle, predicted bytes) of a waiting factorization
        (fresh matrix or refactor of an evicted factor) whose pattern analysis is done, else None."""
        A, key = (req.matrix, self._pattern_key(req.matrix)) if req.kind == "factor_solve" else self._evicted[req.factor_id]
        fut = self._patterns.get(key)
        if fut is None or not fut.done() or fut.exception() is not None:
            return None
        T = fut.result()
        if not req.need:
            req.need = T.PredictDeviceBytes(self.precision, req.nrhs) + ALLOC_SLACK
        return A, key, T, req.need

    def _factor_could_start(self, req: Request) -> bool:
        """A waiting factorization that would start now if a slot were free: its analysis is
        done, its id is not being factored, the factorization cap has room and its predicted
        footprint fits the memory budget."""
        fid = req.factor_id
        if req.kind == "solve" and (fid in self._factors or fid not in self._evicted):
            return False
        if fid in self._pending_ids or self._factor_inflight >= self.max_factor_inflight:
            return False
        got = self._factor_need(req)
        return got is not None and got[3] <= self.memory_budget

    def _admit_pass(self, jobs: list, solves: bool) -> None:
        factor_blocked = False  # a factorization waits for memory: later ones may not pass it
        limit = self.max_inflight
        if solves and any(self._factor_could_start(r) for r in self._waiting):
            limit -= 1  # a factorization ready to start keeps one slot: a stream of solves cannot starve it
        for req in list(self._waiting):
            if self._inflight + len(jobs) >= limit:
                break
            if req not in self._waiting:  # taken by a merged solve group above
                continue
            fid = req.factor_id
            cached_solve = req.kind == "solve" and fid in self._factors
            if solves != cached_solve:
                continue
            if cached_solve:
                F = self._factors[fid]
                if F.busy:
                    continue
                group, cols = [], 0
                for r in self._waiting:
                    if r.kind == "solve" and r.factor_id == fid and cols + r.nrhs <= max(self.max_batch_rhs, req.nrhs):
                        group.append(r)
                        cols += r.nrhs
                need = max(0, F.M.PredictDeviceBytes(self.precision, cols) + ALLOC_SLACK - F.bytes)
                F.busy = True  # protect it from eviction while making room
                if need and not self._evict(need):
                    F.busy = False
                    continue
                F.bytes += need
                self._reserved += need
                self._factors.move_to_end(fid)
                for r in group:
                    self._waiting.remove(r)
                jobs.append(("solve", F, group))
                continue
            if req.kind == "solve" and fid not in self._evicted:
                if fid in self._pending_ids:
                    continue  # its factorization is running
                if not any(r.kind == "factor_solve" and r.factor_id == fid for r in self._waiting):
                    self._waiting.remove(req)
                    req.future.set_exception(KeyError(f"no factor {fid!r}"))
                continue
            # a factorization: fresh matrix, or refactor of an evicted factor
            if factor_blocked or fid in self._pending_ids:
                continue
            if self._factor_inflight + sum(1 for j in jobs if j[0] == "factor") >= self.max_factor_inflight:
                break
            if fid in self._factors:  # same id factored again: drop the old factor once idle
                F = self._factors[fid]
                if F.busy:
                    continue
                del self._factors[fid]
                self._reserved -= F.bytes
                F.M.close()
            A, key = (req.matrix, self._pattern_key(req.matrix)) if req.kind == "factor_solve" else self._evicted[fid]
            if key not in self._patterns:
                self._patterns[key] = self._analysis.submit(self._analyse, A)
                self._patterns[key].add_done_callback(lambda _f: self._notify())
            fut = self._patterns[key]
            if not fut.done():
                continue
            if fut.exception() is not None:
                self._waiting.remove(req)
                req.future.set_exception(fut.exception())
                continue
            _, _, T, need = self._factor_need(req)
            if need > self.memory_budget:  # could never fit: fail now instead of waiting forever
                self._waiting.remove(req)
                req.future.set_exception(MemoryError(
                    f"factor {fid!r} needs {need} device bytes, above the memory budget of {self.memory_budget}"))
                continue
            if not self._evict(need):
                factor_blocked = True
                continue
            self._reserved += need
            self._pending_ids.add(fid)
            self._waiting.remove(req)
            self._evicted.pop(fid, None)
            jobs.append(("factor", req, A, key, T, need))

    # -- workers ----------------------------------------------------------------------
    def _options(self) -> symPACKOptions:
        return symPACKOptions(device=self.device, precision=self.precision, ir_tolerance=self.ir_tolerance)

    def _run(self, job):
        try:
            if job[0] == "factor":
                self._run_factor(*job[1:])
            else:
                self._run_solve(*job[1:])
        finally:
            with self._cv:
                self._inflight -= 1
                if job[0] == "factor":
                    self._factor_inflight -= 1
                self._cv.notify_all()

    def _finish(self, req: Request, x, inf, batched: int):
        req.t_done = time.perf_counter()
        req.batched = batched
        if not req.keep:
            x = None
            req.rhs = None
            req.matrix = None
        res = Result(x=x, backward_error=float(inf.backward_error), ir_iterations=int(inf.ir_iterations),
                     latency_s=req.latency, queue_s=req.t_start - req.t_submit, batched=batched,
                     refactored=req.refactored)
        with self._cv:
            self.done.append(req)
        req.future.set_result(res)

    def _run_factor(self, req: Request, A: DistSparseMatrix, key: str, T: symPACKMatrix2D, need: int):
        req.t_start = time.perf_counter()
        req.refactored = req.kind == "solve"
        M = symPACKMatrix2D()
        try:
            M.Init(self._options())
            M.SymbolicFactorizationFrom(T)
            M.DistributeMatrix(A)
            M.Factorize()
            M.Solve(req.rhs)
            x = M.GetSolution(nrhs=req.nrhs)
            if req.rhs.ndim == 1:
                x = x.reshape(-1)
            inf = M.info()
        except BaseException as e:  # noqa: BLE001 - handed to the caller through the future
            M.close()
            with self._cv:
                self._reserved -= need
                self._pending_ids.discard(req.factor_id)
                self._evicted[req.factor_id] = (A, key)
            req.future.set_exception(e)
            return
        with self._cv:
            F = _Factor(M, need, A, key, A.size)
            F.busy = False
            self._factors[req.factor_id] = F
            self._pending_ids.discard(req.factor_id)
            self.stats["factorizations"] += 1
            self.stats["refactors"] += int(req.refactored)
        self._finish(req, x, inf, 1)

    def _run_solve(self, F: _Factor, group: list[Request]):
        t0 = time.perf_counter()
        for r in group:
            r.t_start = t0
        try:
            B = np.concatenate([r.rhs.reshape(F.n, -1) for r in group], axis=1)
            F.M.Solve(B)
            X = F.M.GetSolution(nrhs=B.shape[1])
            inf = F.M.info()
        except BaseException as e:  # noqa: BLE001
            with self._cv:
                F.busy = False
            for r in group:
                r.future.set_exception(e)
            return
        c = 0
        for r in group:
            x = X[:, c:c + r.nrhs]
            c += r.nrhs
            self._finish(r, x.reshape(-1) if r.rhs.ndim == 1 else np.ascontiguousarray(x), inf, len(group))
        with self._cv:
            F.busy = False
            self.stats["solve_batches"] += 1
            self.stats["solves"] += len(group)


def latency_summary(reqs: list[Request]) -> dict:
    lat = np.array([r.latency for r in reqs]) * 1e3
    if len(lat) == 0:
        return {}
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}


# -- the serving workload: Poisson arrivals of factor+solve and solve-only requests ----------------

class _Pattern:
    """One grid pattern of the request stream and a cheap source of fresh values."""

    def __init__(self, kind: str, k: int, delta: float = 1e-2):
        from . import generators as G
        self.kind, self.k, self.delta = kind, k, delta
        if kind == "st27":
            n, cp, ri, v = G.stencil27(k, k, k, delta, seed=0)
        else:
            n, cp, ri, v = G.laplacian_2d(k, k)
        self.n, self.colptr, self.rowind, self.base = n, cp, ri, v
        self.cols = np.repeat(np.arange(n), np.diff(cp))
        self.rows = ri.astype(np.int64) - 1
        self.diag = self.rows == self.cols

    def matrix(self, seed: int) -> DistSparseMatrix:
        """st27: off-diagonals U[-1, 0) from seed, diagonal |row sum| (1 + delta), as the
        27-point generator draws them; lap2d: the 5-point Laplacian itself."""
        if self.kind != "st27":
            return DistSparseMatrix.from_lower_csc(self.n, self.colptr, self.rowind, self.base)
        rng = np.random.default_rng(seed)
        off = ~self.diag
        v = np.empty(len(self.rows))
        o = -rng.uniform(0.0, 1.0, size=int(off.sum()))
        o[o == 0.0] = -0.5
        v[off] = o
        a = np.abs(o)
        rs = np.bincount(self.rows[off], a, self.n) + np.bincount(self.cols[off], a, self.n)
        v[self.diag] = rs[self.rows[self.diag]] * (1.0 + self.delta)
        return DistSparseMatrix.from_lower_csc(self.n, self.colptr, self.rowind, v)


# Grid ladders of the stream (n from 1,000 to 216,000, about x2 apart): a
# serving workload reuses a modest set of patterns with fresh values.
ST27_GRIDS = (10, 13, 17, 22, 28, 36, 46, 60)
LAP2D_GRIDS = (32, 45, 64, 90, 128, 181, 256, 362, 464)


def request_stream(count: int, rate: float, seed: int = 0, n_min: int = 1000, n_max: int = 216000,
                   factor_frac: float = 0.3, nrhs_max: int = 64, recent: int = 8):
    """Seeded stream of (arrival_s, Request) with Poisson arrivals at `rate` per
    second.  A factor+solve request (probability factor_frac) draws n
    log-uniform in [n_min, n_max] and a generator (27-point stencil, delta
    1e-2, or 2D 5-point Laplacian) and takes the grid of that generator's
    ladder whose size is closest to n; its values are fresh (own seed).  A solve-only request
    targets one of the `recent` latest factors.  nrhs is uniform in
    1..nrhs_max; right-hand sides are standard normal."""
    rng = np.random.default_rng(seed)
    st_k = [k for k in ST27_GRIDS if n_min <= k ** 3 <= n_max] or [ST27_GRIDS[0]]
    lp_k = [k for k in LAP2D_GRIDS if n_min <= k * k <= n_max] or [LAP2D_GRIDS[0]]
    patterns: dict[tuple, _Pattern] = {}
    t, out, factors = 0.0, [], []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        nrhs = int(rng.integers(1, nrhs_max + 1))
        if not factors or rng.uniform() < factor_frac:
            n = np.exp(rng.uniform(np.log(n_min), np.log(n_max)))
            if rng.uniform() < 0.5:
                kind, k = "st27", min(st_k, key=lambda k: abs(np.log(k ** 3 / n)))
            else:
                kind, k = "lap2d", min(lp_k, key=lambda k: abs(np.log(k * k / n)))
            if (kind, k) not in patterns:
                patterns[(kind, k)] = _Pattern(kind, k)
            P = patterns[(kind, k)]
            fid = f"f{i}"
            factors.append((fid, P.n))
            req = Request("factor_solve", fid, None, spec=(P, int(rng.integers(1 << 31)), P.n, nrhs))
        else:
            fid, n = factors[-1 - int(rng.integers(min(recent, len(factors))))]
            req = Request("solve", fid, None, spec=(None, int(rng.integers(1 << 31)), n, nrhs))
        out.append((t, req))
    return out


def materialise(req: Request) -> Request:
    """Draw a stream request's matrix values and right-hand sides from its seed."""
    if req.spec is not None:
        P, seed, n, nrhs = req.spec
        if P is not None:
            req.matrix = P.matrix(seed)
        req.rhs = np.random.default_rng(seed + 1).standard_normal((n, nrhs))
        req.spec = None
    return req


def replay(service: SolverService, stream, time_scale: float = 1.0, timeout: float = 600.0) -> float:
    """Submit the stream at its arrival times (scaled) and wait for all results.
    Returns the wall time from the first arrival to the last completion."""
    t0 = time.perf_counter()
    for t, req in stream:
        materialise(req)
        dt = t0 + t * time_scale - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        service.submit(req)
    service.drain(timeout=timeout)
    return max(r.t_done for _, r in stream) - t0
