"""Host-side mirror of symPACK's ``symPACKMatrix2D`` interface over the C ABI.

Names, argument meaning and call order follow the reference
(include/sympack/symPACKMatrix2D.hpp:2618-2627, symPACKMatrixBase.hpp:51-103,
driver/run_sympack2D.cpp:80-124)::

    opts = symPACKOptions()                      # Types.hpp:106-201
    A = DistSparseMatrix.from_lower_csc(n, colptr, rowind, nzval)   # 1-based lower CSC
    M = symPACKMatrix2D()
    M.Init(opts)
    M.SymbolicFactorization(A)
    M.DistributeMatrix(A)
    M.Factorize()
    M.Solve(rhs, nrhs)                           # rhs column-major n x nrhs
    M.GetSolution(B, nrhs)                       # B receives the solution

Errors: invalid options raise ``ValueError`` (the reference throws
``std::logic_error``, 2D.hpp:2766-2789); a non-SPD pivot raises ``NotSPDError``
(the reference throws "Matrix is not HPD.", lapack.cpp:293-306, then spins).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N


class SymPACKError(RuntimeError):
    """A failed call into the native solver (carries the C status code)."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class NotSPDError(SymPACKError):
    """Non-positive pivot: the matrix is not Hermitian positive definite."""


class StateError(SymPACKError):
    """Methods called out of order (e.g. Solve before Factorize)."""


class DeviceTimeoutError(SymPACKError):
    """A bounded device-side wait expired; the handle remains usable."""


def _raise(code: int, where: str, handle=None):
    if code == N.SPB_OK:
        return
    lib = N.load()
    msg = lib.spb_last_error(handle).decode() if handle else ""
    text = f"{where}: {msg or 'error %d' % code}"
    if code == N.SPB_ERR_NOT_SPD:
        raise NotSPDError(code, text)
    if code == N.SPB_ERR_STATE:
        raise StateError(code, text)
    if code == N.SPB_ERR_TIMEOUT:
        raise DeviceTimeoutError(code, text)
    if code == N.SPB_ERR_INVALID:
        raise ValueError(text)
    raise SymPACKError(code, text)


@dataclass
class RelaxationParameters:
    """Types.hpp:22-96; driver default after SetMaxSize(0) (utils.hpp:342-348)."""

    nrelax0: int = 8
    nrelax1: int = 32
    nrelax2: int = 64
    maxSize: int = 0
    zrelax0: float = 0.8
    zrelax1: float = 0.1
    zrelax2: float = 0.05


@dataclass
class symPACKOptions:
    orderingStr: str = "MMD"
    relax: RelaxationParameters = field(default_factory=RelaxationParameters)
    perm: np.ndarray | None = None      # USER ordering, 1-based new -> old
    precision: str = "FP64"             # "FP64" or "FP32_IR"
    ir_tolerance: float = 1e-12
    ir_max_iter: int = 30
    device: int = 0
    verbose: int = 0
    plan_small_max_w: int = 0      # 0 = library default
    plan_big_tile_rows: int = 0    # 0 = library default
    fp32_engine: str = "tcgen05-tma"  # FP32_IR update tiles: "tcgen05-tma", "tcgen05", "mma.sync",
                                      # "tcgen05-persistent"
    decomposition: str = "LL"      # "LL" (Cholesky) or "LDL" (L D L^T, FP64), the driver's -fact
    plan_outer_nb: int = 0         # columns per outer block of wide panels (0 = library default 256)
    plan_dense_min_w: int = 0      # accepted for compatibility, no effect (the super-block solve replaced it)
    plan_solve_chunk: int = 0      # 64-column blocks per solve super-block (0 = library default 8)
    plan_solve_tiles: int = 0      # 64 x 64 tiles per super-block solve task (0 = library default 2)
    factor_schedule: str = "auto"  # "persistent" (one launch; FP64, or FP32_IR with tcgen05-tma), "steps",
                                   # or "auto" (persistent for FP64, steps for FP32_IR)

    def to_c(self) -> N.spb_options:
        if self.orderingStr not in N.ORDERINGS:
            raise ValueError(
                "This ordering method is not supported by this solver. Valid options are: "
                + " ".join(N.ORDERINGS))
        if self.precision not in N.PRECISIONS:
            raise ValueError(f"unknown precision {self.precision!r}")
        o = N.spb_options()
        N.load().spb_default_options(C.byref(o))
        o.ordering = N.ORDERINGS[self.orderingStr]
        r = self.relax
        o.nrelax0, o.nrelax1, o.nrelax2, o.max_snode = r.nrelax0, r.nrelax1, r.nrelax2, r.maxSize
        o.zrelax0, o.zrelax1, o.zrelax2 = r.zrelax0, r.zrelax1, r.zrelax2
        o.device = self.device
        o.precision = N.PRECISIONS[self.precision]
        o.ir_tolerance = self.ir_tolerance
        o.ir_max_iter = self.ir_max_iter
        o.verbose = self.verbose
        o.plan_small_max_w = self.plan_small_max_w
        o.plan_big_tile_rows = self.plan_big_tile_rows
        o.plan_outer_nb = self.plan_outer_nb
        o.plan_dense_min_w = self.plan_dense_min_w
        o.plan_solve_chunk = self.plan_solve_chunk
        o.plan_solve_tiles = self.plan_solve_tiles
        schedules = {"auto": 0, "steps": 1, "persistent": 2}
        if self.factor_schedule not in schedules:
            raise ValueError(f"unknown factor_schedule {self.factor_schedule!r} (auto, persistent or steps)")
        o.factor_schedule = schedules[self.factor_schedule]
        engines = {"tcgen05": 0, "mma.sync": 1, "tcgen05-persistent": 2, "tcgen05-tma": 3}
        if self.fp32_engine not in engines:
            raise ValueError(f"unknown fp32_engine {self.fp32_engine!r}")
        o.fp32_engine = engines[self.fp32_engine]
        if self.decomposition not in N.DECOMPOSITIONS:
            raise ValueError(f"unknown decomposition {self.decomposition!r} (LL or LDL)")
        o.decomposition = N.DECOMPOSITIONS[self.decomposition]
        return o


@dataclass
class DistSparseMatrix:
    """Lower triangle (diagonal included) of a symmetric matrix, 1-based CSC
    with sorted rows: DistSparseMatrix<T> at one rank (DistSparseMatrix.hpp:49-63)."""

    size: int
    colptr: np.ndarray   # int64, n+1, colptr[0] == 1
    rowind: np.ndarray   # int32, nnz
    nzvalLocal: np.ndarray  # float64, nnz

    @property
    def nnz(self) -> int:
        return int(self.colptr[-1] - 1)

    @classmethod
    def from_lower_csc(cls, n, colptr, rowind, nzval) -> "DistSparseMatrix":
        return cls(int(n), np.ascontiguousarray(colptr, dtype=np.int64),
                   np.ascontiguousarray(rowind, dtype=np.int32),
                   np.ascontiguousarray(nzval, dtype=np.float64))

    @classmethod
    def from_rb(cls, path: str) -> "DistSparseMatrix":
        """ReadMatrix for a Rutherford-Boeing file (utility.hpp:1695-1727)."""
        lib = N.load()
        n = C.c_int32()
        nnz = C.c_int64()
        _raise(lib.spb_rb_info(path.encode(), C.byref(n), C.byref(nnz)), "spb_rb_info")
        colptr = np.empty(n.value + 1, np.int64)
        rowind = np.empty(nnz.value, np.int32)
        nzval = np.empty(nnz.value, np.float64)
        _raise(lib.spb_rb_read(path.encode(), _i64(colptr), _i32(rowind), _d(nzval)), "spb_rb_read")
        return cls(n.value, colptr, rowind, nzval)

    def write_rb(self, path: str, title: str = "") -> None:
        lib = N.load()
        _raise(lib.spb_rb_write(path.encode(), title.encode(), self.size, _i64(self.colptr),
                                _i32(self.rowind), _d(self.nzvalLocal)), "spb_rb_write")

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """y = A x with the symmetric expansion of the stored lower triangle (float64)."""
        n = self.size
        cols = np.repeat(np.arange(n), np.diff(self.colptr)).astype(np.int64)
        rows = self.rowind.astype(np.int64) - 1
        x2 = x.reshape(n, -1)
        y = np.zeros_like(x2, dtype=np.float64)
        np.add.at(y, rows, self.nzvalLocal[:, None] * x2[cols])
        off = rows != cols
        np.add.at(y, cols[off], self.nzvalLocal[off, None] * x2[rows[off]])
        return y.reshape(x.shape)


def _i32(a):
    return a.ctypes.data_as(N._I32P)


def _i64(a):
    return a.ctypes.data_as(N._I64P)


def _d(a):
    return a.ctypes.data_as(N._DP)


def matlab_sparse(n: int, xsuper, xlindx, lindx, panels) -> str:
    """The factor as a MATLAB expression, the form of symPACKMatrix2D::DumpMatlab
    (2D.hpp:6762-6854): ``+sparse([rows],[cols],[values],n,n)`` over the stored entries of
    the lower triangle, supernode by supernode and row by row, in the permuted ordering
    (1-based), values with 17 significant digits.  ``xsuper`` / ``xlindx`` / ``lindx`` are
    the supernodal partition and row structure (1-based) and ``panels`` the factor, per
    supernode its h x w panel column-major with leading dimension h."""
    xsuper = np.asarray(xsuper, np.int64)
    xlindx = np.asarray(xlindx, np.int64)
    lindx = np.asarray(lindx, np.int64)
    panels = np.asarray(panels, np.float64)
    rows, cols, vals = [], [], []
    off = 0
    for s in range(len(xsuper) - 1):
        fc, w = int(xsuper[s]), int(xsuper[s + 1] - xsuper[s])
        r = lindx[xlindx[s] - 1:xlindx[s + 1] - 1]
        h = len(r)
        P = panels[off:off + h * w].reshape(w, h).T  # P[i, j]: row r[i], column fc + j
        off += h * w
        c = fc + np.arange(w)
        keep = r[:, None] >= c[None, :]  # lower triangle (the diagonal block's upper part is not stored)
        ii, jj = np.nonzero(keep)  # row-major: row by row, its columns in order
        rows.append(r[ii])
        cols.append(c[jj])
        vals.append(P[ii, jj])
    rows = np.concatenate(rows) if rows else np.empty(0, np.int64)
    cols = np.concatenate(cols) if cols else np.empty(0, np.int64)
    vals = np.concatenate(vals) if vals else np.empty(0)
    return ("+sparse([" + " ".join(map(str, rows.tolist())) + "],[" + " ".join(map(str, cols.tolist())) + "],["
            + " ".join(f"{v:.16e}" for v in vals.tolist()) + f"],{n},{n})\n")


class symPACKMatrix2D:
    """One supernodal Cholesky factorization held on one GPU."""

    def __init__(self):
        self._lib = N.load()
        self._h = None
        self._n = 0
        self.options: symPACKOptions | None = None

    # -- lifecycle -----------------------------------------------------------
    def Init(self, options: symPACKOptions | None = None) -> None:
        self.options = options or symPACKOptions()
        copt = self.options.to_c()
        perm_buf = None
        if self.options.orderingStr == "USER":
            if self.options.perm is None:
                raise ValueError("When using USER, symPACKOptions.perm must be provided.")
            perm_buf = np.ascontiguousarray(self.options.perm, dtype=np.int32)
            copt.user_perm = _i32(perm_buf)
        self._perm_buf = perm_buf
        self.close()
        h = C.c_void_p()
        _raise(self._lib.spb_create(C.byref(copt), C.byref(h)), "spb_create")
        self._h = h

    def close(self) -> None:
        if self._h:
            self._lib.spb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _need(self):
        if not self._h:
            raise StateError(N.SPB_ERR_STATE, "call Init first")
        return self._h

    # -- reference methods -----------------------------------------------------
    def SymbolicFactorization(self, A: DistSparseMatrix) -> None:
        h = self._need()
        self._n = A.size
        _raise(self._lib.spb_symbolic(h, A.size, _i64(A.colptr), _i32(A.rowind)), "SymbolicFactorization", h)

    def SymbolicFactorizationBatch(self, A: DistSparseMatrix, sys_offsets) -> None:
        """Batching: A is block-diagonal; system k spans rows sys_offsets[k]..sys_offsets[k+1]-1."""
        h = self._need()
        self._n = A.size
        offs = np.ascontiguousarray(sys_offsets, dtype=np.int32)
        _raise(self._lib.spb_symbolic_batch(h, len(offs) - 1, _i32(offs), A.size, _i64(A.colptr), _i32(A.rowind)),
               "SymbolicFactorizationBatch", h)

    def SymbolicFactorizationFrom(self, other: "symPACKMatrix2D") -> None:
        """Reuse other's symbolic analysis (same structure) without ordering again."""
        h = self._need()
        self._n = other._n
        _raise(self._lib.spb_symbolic_from(h, other._need()), "SymbolicFactorizationFrom", h)

    def PredictDeviceBytes(self, precision: str | None = None, nrhs: int = 1) -> int:
        """HBM bytes a factor + solve of nrhs columns needs with this analysis."""
        h = self._need()
        prec = N.PRECISIONS[precision or self.options.precision]
        out = C.c_int64()
        _raise(self._lib.spb_predict_device_bytes(h, prec, int(nrhs), C.byref(out)), "PredictDeviceBytes", h)
        return int(out.value)

    def Replan(self, small_max_w: int = 0, big_tile_rows: int = 0, outer_nb: int = 0) -> None:
        """Rebuild the device plan with other tile shapes (0 = library default); values
        must be distributed again."""
        h = self._need()
        _raise(self._lib.spb_replan(h, int(small_max_w), int(big_tile_rows), int(outer_nb)), "Replan", h)

    def DistributeMatrix(self, A: DistSparseMatrix) -> None:
        h = self._need()
        _raise(self._lib.spb_distribute(h, _d(A.nzvalLocal)), "DistributeMatrix", h)

    def DistributeMatrixDevice(self, d_nzval_ptr: int) -> None:
        """DistributeMatrix from values already resident on the device (pointer)."""
        h = self._need()
        _raise(self._lib.spb_distribute_device(h, C.c_void_p(d_nzval_ptr)), "DistributeMatrix", h)

    def Factorize(self) -> None:
        h = self._need()
        _raise(self._lib.spb_factorize(h), "Factorize", h)

    def Solve(self, RHS: np.ndarray, nrhs: int | None = None) -> None:
        h = self._need()
        rhs = np.asfortranarray(np.asarray(RHS, dtype=np.float64).reshape(self._n, -1, order="F"))
        nrhs = rhs.shape[1] if nrhs is None else nrhs
        _raise(self._lib.spb_solve(h, _d(rhs), nrhs, self._n), "Solve", h)

    def GetSolution(self, B: np.ndarray | None = None, nrhs: int = 1) -> np.ndarray:
        h = self._need()
        out = np.empty((self._n, nrhs), dtype=np.float64, order="F")
        _raise(self._lib.spb_get_solution(h, _d(out), nrhs, self._n), "GetSolution", h)
        if B is not None:
            B.reshape(self._n, -1, order="F")[:, :nrhs] = out
        return out

    def SolveDevice(self, d_rhs_ptr: int, d_x_ptr: int, nrhs: int, ld: int) -> None:
        h = self._need()
        _raise(self._lib.spb_solve_device(h, C.c_void_p(d_rhs_ptr), C.c_void_p(d_x_ptr), nrhs, ld),
               "SolveDevice", h)

    def SetStream(self, stream_handle: int | None) -> None:
        """Run later calls on a caller-owned CUDA stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        _raise(self._lib.spb_set_stream(self._need(), C.c_void_p(stream_handle or 0)), "SetStream", self._h)

    def SetWaitLimit(self, polls: int) -> None:
        """Bound of every device-side wait in the solve kernels (polls ~128 ns apart)."""
        _raise(self._lib.spb_set_wait_limit(self._need(), int(polls)), "SetWaitLimit", self._h)

    def DebugStall(self, supernode: int) -> None:
        """Failure-detection test hook: the forward solve waits for an update nobody sends."""
        _raise(self._lib.spb_debug_stall(self._need(), int(supernode)), "DebugStall", self._h)

    def SetFactorTrace(self, on: bool = True) -> None:
        """Record the per-task timeline of later persistent factorizations."""
        _raise(self._lib.spb_set_factor_trace(self._need(), 1 if on else 0), "SetFactorTrace", self._h)

    def GetFactorTrace(self):
        """(ntasks, 4) uint64 rows {handed out, dependencies met, done (ns), SM} in dispatch
        order, and the task kinds (0 small, 1 diagonal block, 2 TRSM, 3 64 x 64 tile, 4 tensor-core tile:
        128 x 64 in FP64, 128 x 128 in FP32)."""
        h = self._need()
        nt = C.c_int64()
        _raise(self._lib.spb_get_factor_trace(h, None, 0, C.byref(nt), None), "GetFactorTrace", h)
        out = np.zeros((nt.value, 4), np.uint64)
        kinds = np.zeros(nt.value, np.int32)
        _raise(self._lib.spb_get_factor_trace(h, out.ctypes.data_as(C.POINTER(C.c_uint64)), nt.value, C.byref(nt),
                                              kinds.ctypes.data_as(C.POINTER(C.c_int32))), "GetFactorTrace", h)
        return out, kinds

    def ReorderFactorFromTrace(self) -> None:
        """Re-order the persistent factorization's tasks by the durations the last traced
        factorization measured (spb_reorder_factor_from_trace)."""
        h = self._need()
        _raise(self._lib.spb_reorder_factor_from_trace(h), "ReorderFactorFromTrace", h)

    def TuneFactorOrder(self, A: "DistSparseMatrix", passes: int = 2) -> list:
        """Profile-guided task order: ``passes`` times, factor A with the task timeline on
        and re-order the tasks by their measured durations.  Leaves A distributed, ready
        for Factorize, and the trace off.  Returns the ordering simulation's predicted
        makespan (microseconds) after each pass."""
        pred = []
        self.SetFactorTrace(True)
        try:
            for _ in range(passes):
                self.DistributeMatrix(A)
                self.Factorize()
                self.ReorderFactorFromTrace()
                pred.append(float(self.info().factor_sched_us))
        finally:
            self.SetFactorTrace(False)
        self.DistributeMatrix(A)
        return pred

    def DebugStallFactor(self, supernode: int) -> None:
        """Failure-detection test hook: the persistent factorization waits for an update nobody sends."""
        _raise(self._lib.spb_debug_stall_factor(self._need(), int(supernode)), "DebugStallFactor", self._h)

    def SetProfiling(self, on: bool = True) -> None:
        _raise(self._lib.spb_set_profiling(self._need(), 1 if on else 0), "SetProfiling", self._h)

    def GetSolveTrace(self, sweep: int = 0) -> np.ndarray:
        """Task timeline of the last profiled solve: (ntasks, 4) uint64 rows
        {grabbed_ns, ready_ns, done_ns, supernode << 8 | kind} (sweep 0 forward, 1 backward)."""
        h = self._need()
        nt = C.c_int64()
        _raise(self._lib.spb_get_solve_trace(h, sweep, None, 0, C.byref(nt)), "GetSolveTrace", h)
        out = np.zeros((nt.value, 4), np.uint64)
        _raise(self._lib.spb_get_solve_trace(h, sweep, out.ctypes.data_as(C.POINTER(C.c_uint64)), nt.value,
                                             C.byref(nt)), "GetSolveTrace", h)
        return out

    def GetProfile(self) -> dict:
        p = N.spb_profile()
        _raise(self._lib.spb_get_profile(self._need(), C.byref(p)), "GetProfile", self._h)
        return {name: dict(ms=p.ms[i], flops=p.flops[i], bytes=p.bytes[i], launches=p.launches[i])
                for i, name in enumerate(N.KIND_NAMES)}

    # -- accessors (symPACKMatrixBase.hpp:96-103) ------------------------------
    def info(self) -> N.spb_info:
        h = self._need()
        inf = N.spb_info()
        _raise(self._lib.spb_get_info(h, C.byref(inf)), "info", h)
        return inf

    def GetOrdering(self):
        n = self._n
        perm = np.empty(n, np.int32)
        invp = np.empty(n, np.int32)
        _raise(self._lib.spb_get_ordering(self._need(), _i32(perm), _i32(invp)), "GetOrdering", self._h)
        return perm, invp

    def GetMMDInvp(self):
        invp = np.empty(self._n, np.int32)
        _raise(self._lib.spb_get_mmd_invp(self._need(), _i32(invp)), "GetMMDInvp", self._h)
        return invp

    def GetETree(self):
        p = np.empty(self._n, np.int32)
        _raise(self._lib.spb_get_etree(self._need(), _i32(p)), "GetETree", self._h)
        return p

    def GetColCounts(self):
        a = np.empty(self._n, np.int32)
        b = np.empty(self._n, np.int32)
        _raise(self._lib.spb_get_colcounts(self._need(), _i32(a), _i32(b)), "GetColCounts", self._h)
        return a, b

    def GetSupernodalPartition(self):
        inf = self.info()
        xs = np.empty(inf.nsuper + 1, np.int32)
        _raise(self._lib.spb_get_supernodes(self._need(), _i32(xs), None), "GetSupernodalPartition", self._h)
        return xs

    def GetSupMembership(self):
        sm = np.empty(self._n, np.int32)
        _raise(self._lib.spb_get_supernodes(self._need(), None, _i32(sm)), "GetSupMembership", self._h)
        return sm

    def GetStructure(self):
        inf = self.info()
        xl = np.empty(inf.nsuper + 1, np.int64)
        li = np.empty(inf.lindx_size, np.int32)
        _raise(self._lib.spb_get_structure(self._need(), _i64(xl), _i32(li)), "GetStructure", self._h)
        return xl, li

    def GetCells(self):
        inf = self.info()
        nc, nb = inf.ncells, inf.nblocks
        arrs = [np.empty(nc, np.int32) for _ in range(5)] + [np.empty(nb, np.int32) for _ in range(2)]
        _raise(self._lib.spb_get_cells(self._need(), *[_i32(a) for a in arrs]), "GetCells", self._h)
        keys = ["I", "K", "nrows", "first_block", "nblocks", "block_first_row", "block_nrows"]
        return dict(zip(keys, arrs))

    def GetFactor(self) -> np.ndarray:
        """Factor panels: per supernode h x w column-major (ld h), upper diagonal block zeroed."""
        xs = self.GetSupernodalPartition()
        xl, _ = self.GetStructure()
        total = int(np.sum((xl[1:] - xl[:-1]) * (xs[1:] - xs[:-1])))
        out = np.empty(total, np.float64)
        _raise(self._lib.spb_get_factor(self._need(), _d(out)), "GetFactor", self._h)
        return out

    def DumpMatlab(self, file=None) -> None:
        """symPACKMatrix2D::DumpMatlab (2D.hpp:6762-6854): write the factor as
        ``+sparse([rows],[cols],[values],n,n)`` (see ``matlab_sparse``) to ``file`` (a path
        or a text stream; default standard output) after Factorize."""
        import sys
        xl, li = self.GetStructure()
        text = matlab_sparse(self._n, self.GetSupernodalPartition(), xl, li, self.GetFactor())
        if file is None:
            sys.stdout.write(text)
        elif isinstance(file, (str, bytes)) or hasattr(file, "__fspath__"):
            with open(file, "w") as f:
                f.write(text)
        else:
            file.write(text)

    # symPACKMatrixMeta accessors (symPACKMatrixBase.hpp:96-103)
    def Size(self) -> int:
        """Order of the analysed matrix (iSize_)."""
        return self._n

    def GetOptions(self) -> "symPACKOptions | None":
        """The options given to Init."""
        return self.options

    def TotalSupernodeCnt(self) -> int:
        """Number of supernodes (0 before the symbolic factorization)."""
        return int(self.info().nsuper) if self._h and self._n else 0

    def GetStatus(self):
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        _raise(self._lib.spb_get_status(self._need(), C.byref(a), C.byref(b), C.byref(c)), "GetStatus", self._h)
        return a.value, b.value, c.value
