/*
 * sympack_b200.h — C ABI of the B200-native supernodal Cholesky factor / solve.
 *
 * The reference (symPACK v2.0) exposes its solver only as the C++ template
 * class symPACKMatrix2D<Ptr, Idx, T> (include/sympack/symPACKMatrix2D.hpp:2618-2627,
 * base interface include/sympack/symPACKMatrixBase.hpp:51-63).  Its only extern "C"
 * functions are symPACK_Init / symPACK_Finalize / symPACK_Rank / symPACK_cuda_setup
 * (include/sympack.hpp:25-36).  Each entry point below replaces one method of that
 * class one-for-one, with plain pointers and sizes so that a ctypes / cgo / JNI
 * binding needs no C++ types:
 *
 *   spb_create            symPACKMatrix2D::Init(symPACKOptions&)               2D.hpp:2649
 *   spb_symbolic          symPACKMatrix2D::SymbolicFactorization(DistSparseMatrix&) 2D.hpp:2699
 *   spb_distribute        symPACKMatrix2D::DistributeMatrix(DistSparseMatrix&)  2D.hpp:6337
 *   spb_factorize         symPACKMatrix2D::Factorize()                          2D.hpp:6579
 *   spb_solve             symPACKMatrix2D::Solve(T* RHS, int nrhs, int rhs_size) 2D.hpp:6643
 *   spb_get_solution      symPACKMatrix2D::GetSolution(T* B, int nrhs)          2D.hpp:6713
 *   spb_get_ordering      symPACKMatrixBase::GetOrdering()                      symPACKMatrixBase.hpp:96-103
 *   spb_get_supernodes    symPACKMatrixBase::GetSupernodalPartition() / GetSupMembership()
 *   spb_get_etree         symPACKMatrixBase::GetETree()
 *
 * Conventions (same as the reference): the input matrix is the lower triangle,
 * diagonal included, in 1-based compressed-column form with rows sorted per
 * column (DistSparseMatrix<T>, DistSparseMatrix.hpp:49-63); right-hand sides and
 * solutions are column-major n x nrhs in the ORIGINAL ordering.  Solve keeps the
 * solution inside the handle until GetSolution copies it out.
 *
 * Errors are status codes instead of exceptions / spins: a non-SPD pivot (where
 * the reference throws "Matrix is not HPD." and then spins in gdb_lock,
 * 2D.hpp:1097-1100) returns SPB_ERR_NOT_SPD with the failing supernode and
 * column available from spb_get_status.
 *
 * A handle owns all of its device memory and one CUDA stream; it is not
 * thread-safe.  All host pointers are read or written synchronously.
 */
#ifndef SYMPACK_B200_H
#define SYMPACK_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPB_OK 0
#define SPB_ERR_INVALID (-1)   /* bad argument or malformed matrix */
#define SPB_ERR_NOT_SPD (-2)   /* non-positive pivot during Factorize */
#define SPB_ERR_OOM (-3)       /* device allocation failed */
#define SPB_ERR_CUDA (-4)      /* any other CUDA runtime failure */
#define SPB_ERR_STATE (-5)     /* call out of order (e.g. Solve before Factorize) */
#define SPB_ERR_STRUCTURE (-6) /* inconsistent symbolic structure detected on the device */
#define SPB_ERR_TIMEOUT (-7)   /* a bounded device wait expired */
#define SPB_ERR_NOT_CONVERGED (-8) /* iterative refinement did not reach its tolerance */

#define SPB_ORDERING_MMD 0
#define SPB_ORDERING_NATURAL 1
#define SPB_ORDERING_USER 2
#define SPB_ORDERING_RCM 3        /* reverse Cuthill-McKee (genrcm.F) */
#define SPB_ORDERING_AMD 4        /* approximate minimum degree (amdbar.F) */

#define SPB_DECOMPOSITION_LL 0    /* A = L L^T (Cholesky, DecompositionType::LL, "-fact LL") */
#define SPB_DECOMPOSITION_LDL 1   /* A = L D L^T without pivoting (DecompositionType::LDL, "-fact LDL"):
                                     symmetric matrices with nonzero pivots in the chosen ordering,
                                     e.g. quasi-definite ones; FP64 only; spb_get_factor returns L with
                                     D on the diagonal; a zero pivot gives SPB_ERR_NOT_SPD */
#define SPB_PRECISION_FP64 0      /* plain FP64 factor and solve (the drop-in path) */
#define SPB_PRECISION_FP32_IR 1   /* FP32 factor + FP64 iterative refinement */

typedef struct spb_handle spb_handle;

/* Mirrors the symPACKOptions fields this path uses (Types.hpp:106-201). */
typedef struct spb_options {
  int ordering;            /* SPB_ORDERING_* ("-ordering", default MMD) */
  int nrelax0, nrelax1, nrelax2; /* supernode relaxation sizes (8, 32, 64) */
  int max_snode;           /* "-b": maximum supernode width, 0 = unlimited (driver default) */
  double zrelax0, zrelax1, zrelax2; /* relaxation zero fractions (0.8, 0.1, 0.05) */
  const int32_t* user_perm; /* SPB_ORDERING_USER: 1-based new->old permutation */
  int device;              /* CUDA device ordinal; < 0 = host-only handle (symbolic analysis only) */
  int precision;           /* SPB_PRECISION_* */
  double ir_tolerance;     /* backward-error target of refinement (1e-12) */
  int ir_max_iter;         /* refinement iteration cap */
  int verbose;
  int plan_small_max_w;    /* widest supernode factored whole in shared memory (0 = default 32) */
  int plan_big_tile_rows;  /* products with this many rows use 128 x 128 tensor-core tiles (0 = default 128) */
  int fp32_engine;         /* FP32_IR 128 x 128 update tiles: 3 = tcgen05 with its operands loaded by
                              TMA from split (hi / lo) copies of the panels, one tensor map per panel
                              with such tiles (spb_default_options; the copies double the FP32 arena's
                              footprint); 0 = tcgen05 with operands staged by cp.async and split per
                              tile (no copies); 1 = mma.sync; 2 = a persistent tcgen05 variant (two
                              accumulators, epilogue warps overlapped with the next tile) */
  int decomposition;       /* SPB_DECOMPOSITION_* (symPACKOptions::decomposition, Types.hpp:97,119) */
  int plan_outer_nb;       /* columns per outer block of a wide panel: its trailing columns are
                              updated once per outer block (0 = default 256; multiple of 64, <= 4096) */
  int plan_dense_min_w;    /* no effect (a former cluster solve of the root, replaced by the
                              super-block solve); kept for layout */
  int plan_solve_chunk;    /* 64-column blocks per solve super-block: a supernode wider than one block
                              is solved through the inverses of its diagonal super-blocks (0 = default 8) */
  int plan_solve_tiles;    /* 64 x 64 tiles per super-block solve task (0 = default 2) */
  int factor_schedule;     /* SPB_FACTOR_PERSISTENT runs every task of the factorization in one
                              persistent launch ordered by dependency counters (FP64, and the FP32
                              form with fp32_engine 3); SPB_FACTOR_STEPS runs the level-ordered launch
                              sequence replayed from a CUDA graph (the FP32 form with engines 0-2
                              always does); SPB_FACTOR_AUTO (0, the default) is persistent for FP64
                              and steps for the FP32 form */
} spb_options;

#define SPB_FACTOR_AUTO 0
#define SPB_FACTOR_STEPS 1
#define SPB_FACTOR_PERSISTENT 2

typedef struct spb_info {
  int32_t n;
  int32_t nsuper;
  int32_t nlevels;         /* height of the supernodal elimination tree */
  int32_t max_width;
  int64_t nnz_a;           /* entries of the input lower triangle */
  int64_t nnz_l;           /* sum of column counts (reference "NNZ in L factor") */
  int64_t lindx_size;      /* total row-structure entries */
  int64_t arena_bytes;     /* device bytes of the factor panels */
  int64_t device_bytes;    /* all device bytes held by the handle */
  double flops_stat;       /* sum of column counts squared (reference "Flops" statistic) */
  double flops_exec;       /* flops the kernel sequence executes */
  int32_t ncells;          /* reference 2D cells (K, I) */
  int32_t nblocks;         /* reference contiguous-row blocks */
  int32_t ir_iterations;   /* refinement steps of the last solve */
  int32_t factor_launches; /* kernels of one factorization (1 for the persistent schedule) */
  double backward_error;   /* componentwise-free backward error of the last solve, if computed */
  int32_t dense_root_width; /* always 0 (a former cluster solve of the root; kept for layout) */
  int32_t pad_;
  int64_t inverse_bytes;    /* device bytes of the diagonal super-block inverses of one operand */
  double factor_sched_us;   /* makespan the persistent factorization's ordering simulation predicts */
  int32_t factor_tasks;     /* tasks of the persistent factorization */
  int32_t pad2_;
} spb_info;

void spb_default_options(spb_options* opt);
int spb_create(const spb_options* opt, spb_handle** out);
void spb_destroy(spb_handle* h);
const char* spb_last_error(const spb_handle* h);

/* SymbolicFactorization: structure only (values not needed). */
int spb_symbolic(spb_handle* h, int32_t n, const int64_t* colptr, const int32_t* rowind);
/* Batching (no counterpart in the reference, which factors one matrix per
 * symPACKMatrix2D object): nsys independent SPD systems given as one
 * block-diagonal lower CSC; system k owns rows and columns
 * sys_offsets[k] .. sys_offsets[k+1]-1 (0-based, sys_offsets[0] = 0,
 * sys_offsets[nsys] = n).  Each system gets its own symbolic analysis, exactly
 * as spb_symbolic would compute it (run in parallel host threads); the analyses
 * are merged into one forest, so distribute / factorize / solve then handle
 * every system of an elimination-tree level in the same launches.  Right-hand
 * sides are the systems' right-hand sides stacked in the same order. */
int spb_symbolic_batch(spb_handle* h, int32_t nsys, const int32_t* sys_offsets, int32_t n, const int64_t* colptr,
                       const int32_t* rowind);
/* Symbolic-analysis reuse (no counterpart in the reference): give h the
 * analysis of src (same structure; any handle, host-only included) without
 * running the ordering again, then set up h's device buffers.  Ordering and
 * relaxation options of the two handles must agree; precision may differ.
 * The serving loop uses it to factor fresh values on a known pattern. */
int spb_symbolic_from(spb_handle* h, const spb_handle* src);
/* HBM footprint a handle with this analysis needs for factor + a solve of nrhs
 * right-hand sides in the given precision (bytes requested from the device
 * allocator).  Works on host-only handles after spb_symbolic. */
int spb_predict_device_bytes(const spb_handle* h, int32_t precision, int32_t nrhs, int64_t* bytes);
/* Rebuild the device plan of the current analysis with other tile shapes
 * (0 = default): supernodes up to small_max_w columns (<= 64) are factored
 * whole in shared memory; update products with at least big_tile_rows rows use
 * 128 x 128 tensor-core tiles.  The symbolic analysis is kept; values must be
 * distributed again.  Used by the tile-shape autotuner. */
int spb_replan(spb_handle* h, int32_t small_max_w, int32_t big_tile_rows, int32_t outer_nb);
/* DistributeMatrix: values in the same order as rowind (host or device pointer). */
int spb_distribute(spb_handle* h, const double* nzval);
int spb_distribute_device(spb_handle* h, const double* d_nzval);
/* Factorize. */
int spb_factorize(spb_handle* h);
/* Solve: host RHS (column-major, leading dimension ldb >= n); the solution stays in the handle. */
int spb_solve(spb_handle* h, const double* rhs, int32_t nrhs, int64_t ldb);
/* GetSolution: copy the last solution to host B (column-major, leading dimension ldb). */
int spb_get_solution(spb_handle* h, double* B, int32_t nrhs, int64_t ldb);
/* Solve with device-resident right-hand sides and solution (both n x nrhs, leading dimension ld). */
int spb_solve_device(spb_handle* h, const double* d_rhs, double* d_x, int32_t nrhs, int64_t ld);

/* Allocation-free variant of spb_solve_device.  No counterpart in the
 * reference (which has no device-side solve entry point at all).
 * For callers that cannot allocate device memory at solve time: services that
 * reserve their whole device-memory budget at start-up (another allocator, such
 * as a framework's caching allocator, owns the rest of the GPU, so a cudaMalloc
 * in the middle of a request could fail), and latency-critical callers, for
 * which cudaMalloc / cudaFree may synchronize the device and stall the work of
 * other streams.  spb_solve_device may grow its workspace with cudaMalloc on a
 * call with more right-hand sides than before; this entry point calls no
 * cudaMalloc, cudaFree or allocating library routine: its scratch (the permuted
 * right-hand sides, the forward solution and the dependency counters) lives in
 * one static __device__ array of 65 MiB that every GPU which loads the library
 * holds until the process exits.
 * Limits: n * nrhs <= 4,194,304, and 2 + 3 * nsuper + 2 * (number of
 * 64-column blocks over all supernodes) <= 262,144 dependency counters;
 * larger requests return SPB_ERR_INVALID with a message saying so.
 * The first call on a device resolves the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * Every call on a device shares the array: calls whose work overlaps on the GPU
 * (other handles or streams) race, so serialize them.  The counters are cleared
 * on every call (and for every 64 right-hand sides); nothing else is kept
 * between calls.  The first call after a factorization also computes the
 * factor's diagonal super-block inverses, in memory the handle allocated with
 * its analysis.  Like spb_solve_device, the call reads the device status word
 * back before it returns, so it waits for the handle's stream. */
int spb_solve_device_noalloc(spb_handle* h, const double* d_rhs, double* d_x, int32_t nrhs, int64_t ld);

/* Introspection for parity checks (arrays sized from spb_get_info). */
int spb_get_info(spb_handle* h, spb_info* info);
int spb_get_ordering(spb_handle* h, int32_t* perm, int32_t* invp);           /* n each, 1-based */
int spb_get_mmd_invp(spb_handle* h, int32_t* invp);                          /* n, before postordering */
int spb_get_etree(spb_handle* h, int32_t* parent);                           /* n, postordered, 0 = root */
int spb_get_colcounts(spb_handle* h, int32_t* cc_fund, int32_t* cc_relaxed); /* n each */
int spb_get_supernodes(spb_handle* h, int32_t* xsuper, int32_t* supmember);  /* nsuper+1, n */
int spb_get_structure(spb_handle* h, int64_t* xlindx, int32_t* lindx);       /* nsuper+1, lindx_size */
/* Cells (K, I) in the reference's construction order and their row blocks. */
int spb_get_cells(spb_handle* h, int32_t* cell_I, int32_t* cell_K, int32_t* cell_nrows,
                  int32_t* cell_first_block, int32_t* cell_nblocks, int32_t* block_first_row,
                  int32_t* block_nrows);
/* Factor: per supernode, the h x w panel column-major with leading dimension h,
 * entries above the diagonal of the diagonal block set to zero.  Size = sum h*w. */
int spb_get_factor(spb_handle* h, double* out);
/* Status of the last factorization: code, supernode (0-based), column (0-based, permuted). */
int spb_get_status(spb_handle* h, int32_t* code, int32_t* supernode, int32_t* column);

/* Bound on every device-side wait of the persistent solve and factorization
 * kernels, in polls about 128 ns apart (default 2^24, a couple of seconds).  A wait
 * that runs out records a timeout; the call returns SPB_ERR_TIMEOUT and the context
 * stays usable. */
int spb_set_wait_limit(spb_handle* h, int64_t polls);
/* Test hook for failure detection: make the forward solve expect one more
 * incoming update for `supernode` than any task delivers (its wait then runs
 * out); -1 restores the true counts. */
int spb_debug_stall(spb_handle* h, int32_t supernode);
/* Test hook for failure detection: make the persistent factorization wait for one
 * more external update into `supernode` than any task delivers; -1 restores. */
int spb_debug_stall_factor(spb_handle* h, int32_t supernode);
/* Per-task timeline of the persistent factorization (analysis): after
 * spb_set_factor_trace(h, 1) every factorization records, per task in dispatch
 * order, {handed out, dependencies met, done} (ns, globaltimer) and the SM;
 * spb_get_factor_trace copies 4 * ntasks values and the task kinds
 * (0 small panel, 1 diagonal block, 2 TRSM tile, 3 64 x 64 tile, 4 128 x 128 tile). */
int spb_set_factor_trace(spb_handle* h, int32_t on);
int spb_get_factor_trace(spb_handle* h, uint64_t* out, int64_t cap, int64_t* ntasks, int32_t* kinds);
/* Profile-guided task order of the persistent factorization: after a factorization
 * traced with spb_set_factor_trace(h, 1), re-order the tasks by the same list scheduling
 * with each task's measured duration in place of the cost model (the plan's
 * factor_sched_us becomes the new prediction).  Later factorizations of this handle use
 * the new order; the tasks, their dependencies and the results do not change.
 * SPB_ERR_STATE without a fresh trace or when the persistent schedule is not in use. */
int spb_reorder_factor_from_trace(spb_handle* h);
/* Reset the device status word (after a reported failure). */
int spb_clear_status(spb_handle* h);

/* Run every later call of this handle on the caller's CUDA stream (a
 * cudaStream_t passed as void*; NULL returns to the handle's own stream).  Calls
 * still return only when their work is complete. */
int spb_set_stream(spb_handle* h, void* stream);

/* Profiling: with profiling on, spb_factorize launches its steps eagerly with a
 * CUDA event pair around each launch, and spb_solve / spb_solve_device time each
 * sweep; spb_get_profile returns per kernel kind the device milliseconds of the
 * last profiled call, the launches, and the algorithmic flops (factor kinds) or
 * bytes (solve kinds: every panel element read once per sweep). */
#define SPB_KIND_ASSEMBLE 0
#define SPB_KIND_FACTOR_SMALL 1
#define SPB_KIND_POTRF_DIAG 2
#define SPB_KIND_TRSM_ROWS 3
#define SPB_KIND_GEMM_SIMT 4
#define SPB_KIND_GEMM_DMMA 5
#define SPB_KIND_SOLVE_FORWARD 6
#define SPB_KIND_SOLVE_BACKWARD 7
#define SPB_KIND_SOLVE_INVERSE 8  /* diagonal super-block inverses (first solve after a factorization) */
#define SPB_KIND_COUNT 9
typedef struct spb_profile {
  double ms[SPB_KIND_COUNT];
  double flops[SPB_KIND_COUNT];
  double bytes[SPB_KIND_COUNT];
  int32_t launches[SPB_KIND_COUNT];
} spb_profile;
int spb_set_profiling(spb_handle* h, int on);
/* Timeline of the last profiled solve's sweep (0 forward, 1 backward), in task
 * order: per task {grabbed, dependencies met, done} in device nanoseconds and
 * (supernode << 8 | task kind).  Copies min(cap, ntasks) tasks; *ntasks gets
 * the sweep's task count (out may be null to query it). */
int spb_get_solve_trace(spb_handle* h, int32_t sweep, uint64_t* out, int64_t cap, int64_t* ntasks);
int spb_get_profile(spb_handle* h, spb_profile* out);

/* Rutherford-Boeing input boundary, replacing ReadMatrix / ReadHB_PARA
 * (include/sympack/utility.hpp:1274-1481, 1695-1727) for one rank.  spb_rb_info
 * reports the size; spb_rb_read fills colptr (n+1), rowind (nnz) and, if not
 * NULL, nzval (nnz), each column's rows sorted.  spb_rb_write writes a real
 * symmetric ("rsa") lower-triangle file in the (8I10) / (4E20.12) layout that
 * reader expects. */
int spb_rb_info(const char* path, int32_t* n, int64_t* nnz);
int spb_rb_read(const char* path, int64_t* colptr, int32_t* rowind, double* nzval);
int spb_rb_write(const char* path, const char* title, int32_t n, const int64_t* colptr, const int32_t* rowind,
                 const double* nzval);

#ifdef __cplusplus
}
#endif

#endif /* SYMPACK_B200_H */
