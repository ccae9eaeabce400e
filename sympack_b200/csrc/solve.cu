// Persistent supernodal triangular solves (sm_100a).
//
// Numerics of symPACK's solve tasks (symPACKMatrix2D.hpp):
//   FUC(J,J): Y_J <- L_JJ^-1 Y_J               (forward_update_contrib, 1519-1527)
//   FUC(K,J): Y_K[rows] -= L_KJ Y_J            (1589-1592)
//   BUC(J,I): X_I -= L_JI^T X_J[rows]           (back_update_contrib, 1741-1744)
//   BUC(I,I): X_I <- L_II^-T X_I                (_tri_solve, 1659-1721)
// The reference's FUC/BUC task graph (5167-5251, 5728-6322) becomes one
// persistent launch per sweep: CTAs take tasks from an atomic counter in a
// topological order (every dependency of a task was handed out earlier, so a
// waiting CTA only ever waits on CTAs that are already running) and
// synchronise through counters in global memory.  Every wait is bounded; on
// expiry the kernel records SPB timeout status and all CTAs leave.
//
// A supernode wider than one 64-column block is split into super-blocks of sb
// blocks.  The diagonal triangle of a super-block is applied through its
// inverse (k_sb_inverse, once per factorization), so the sb dependent block
// solves of a substitution become sb independent row-block products: the chain
// of a wide supernode has two steps per super-block (its DI products, then the
// updates of the next super-block) instead of one per 64 columns.  The forward
// sweep reads the permuted right-hand sides Y (accumulating the descendants'
// contributions there) and writes its solution to Z; the backward sweep
// accumulates into Z and writes the final solution X.
#include "kernels.cuh"

namespace spb {
namespace dev {

namespace {

constexpr int kT = 64;         // rows / columns per task unit
constexpr int kPld = 65;       // padded leading dimension of a staged 64 x 64 tile
constexpr int kThreads = 256;
// staged tile (64 x 65), right-hand-side staging (64 x 64), and the accumulator of kR
// right-hand sides; kR = 16 keeps three CTAs per SM
template <int kR>
constexpr size_t solve_smem() { return (size_t)(kT * kPld + kT * kT + kT * kR) * sizeof(double); }
template <int kR>
constexpr int solve_min_blocks() { return kR <= 16 ? 3 : 2; }

__device__ __forceinline__ void report_status(Status* st, int code, int s, int col) {
  if (atomicCAS(&st->code, 0, code) == 0) {
    st->supernode = s;
    st->column = col;
  }
}

__device__ __forceinline__ int ld_acquire(const int32_t* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Counter increment with release semantics: after a barrier, a thread's release
// publishes the whole block's earlier writes to any thread that acquires the counter.
__device__ __forceinline__ void red_release(int32_t* p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int status_code(const Status* st) { return *(volatile const int32_t*)&st->code; }

// Block-wide: wait until *flag >= target (thread 0 polls with acquire loads; the
// barrier then orders every thread's later reads after the acquire).  False on
// timeout or if another CTA has already recorded a failure.
__device__ bool wait_geq(const int32_t* flag, int target, Status* st, int s, int* sh_ok, long long limit) {
  if (threadIdx.x == 0) {
    int good = 1;
    if (ld_acquire(flag) < target) {
      good = 0;
      for (long long it = 0; it < limit; ++it) {
        if (it >= 256) __nanosleep(128);  // short waits poll back to back (each poll is an L2 round trip)
        if (ld_acquire(flag) >= target) {
          good = 1;
          break;
        }
        if (status_code(st) != 0) break;
      }
      if (!good && status_code(st) == 0) report_status(st, 3, s, target);
    }
    *sh_ok = good;
  }
  __syncthreads();
  int r = *sh_ok;
  __syncthreads();
  return r != 0;
}

// A 64 x 64 tile of T (column-major, leading dimension ld; rows < m and columns < kk
// valid, zero elsewhere) held in registers, 16 entries per thread, so that the next
// tile's loads are in flight while the current one is used.
template <class T>
struct TileRegs {
  static constexpr int kPer = kT * kT / kThreads;
  T v[kPer];
  __device__ __forceinline__ void load(const T* P, int64_t ld, int m, int kk) {
    if (m == kT && kk == kT) {
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        const int idx = threadIdx.x + q * kThreads, k = idx >> 6, r = idx & 63;
        v[q] = P[r + (int64_t)k * ld];
      }
      return;
    }
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      const int idx = threadIdx.x + q * kThreads, k = idx >> 6, r = idx & 63;
      v[q] = (r < m && k < kk) ? P[r + (int64_t)k * ld] : T(0);
    }
  }
  __device__ __forceinline__ void store(double* A) const {
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      const int idx = threadIdx.x + q * kThreads, k = idx >> 6, r = idx & 63;
      A[r + k * kPld] = (double)v[q];
    }
  }
};

// Stage L rows [r0, r0+m) x columns [c0, c0+kk) of a panel into A (ld kPld), widened to FP64.
template <class T, int kLd = kPld>
__device__ __forceinline__ void stage_block(double* A, const T* P, int64_t ld, int r0, int m, int c0, int kk) {
  if (m == kT && kk == kT) {
    T v[kT * kT / kThreads];
#pragma unroll
    for (int q = 0; q < kT * kT / kThreads; ++q) {
      const int idx = threadIdx.x + q * kThreads, k = idx / kT, r = idx - k * kT;
      v[q] = P[(r0 + r) + (int64_t)(c0 + k) * ld];
    }
#pragma unroll
    for (int q = 0; q < kT * kT / kThreads; ++q) {
      const int idx = threadIdx.x + q * kThreads, k = idx / kT, r = idx - k * kT;
      A[r + k * kLd] = (double)v[q];
    }
    return;
  }
  for (int idx = threadIdx.x; idx < m * kk; idx += kThreads) {
    int k = idx / m, r = idx - k * m;
    A[r + k * kLd] = (double)P[(r0 + r) + (int64_t)(c0 + k) * ld];
  }
}

// Stage X rows x0.. (contiguous) or rows rl[0..] (gathered) into B (leading dimension
// ldb), through L2.
__device__ __forceinline__ void stage_x(double* B, int ldb, const double* X, int64_t ldx, int x0, const int32_t* rl,
                                        int m, int nr) {
  for (int idx = threadIdx.x; idx < m * nr; idx += kThreads) {
    int c = idx / m, r = idx - c * m;
    int row = rl ? rl[r] : x0 + r;
    B[r + c * ldb] = __ldcg(X + row + c * ldx);
  }
}

// acc[i + c*kT] += sum_{k < kk} A(i, k) B[k + c*ldb]  for i < m, c < nr, with
// A(i, k) = A[i + k*kPld] (kTrans false) or A[k + i*kPld] (kTrans true).  Few outputs
// (one right-hand side): four threads per output and a shuffle reduction.
template <bool kTrans>
__device__ __forceinline__ void tile_gemv(double* acc, const double* A, const double* B, int ldb, int m, int kk,
                                          int nr) {
  if (m * nr * 4 <= kThreads) {
    const int idx = threadIdx.x >> 2, part = threadIdx.x & 3;
    const int c = idx / m, i = idx - c * m;
    double s = 0.0;
    if (idx < m * nr)
      for (int k = part; k < kk; k += 4) s = fma(kTrans ? A[k + i * kPld] : A[i + k * kPld], B[k + c * ldb], s);
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if (idx < m * nr && part == 0) acc[i + c * kT] += s;
    return;
  }
  for (int idx = threadIdx.x; idx < m * nr; idx += kThreads) {
    const int c = idx / m, i = idx - c * m;
    double s = 0.0;
    for (int k = 0; k < kk; ++k) s = fma(kTrans ? A[k + i * kPld] : A[i + k * kPld], B[k + c * ldb], s);
    acc[i + c * kT] += s;
  }
}

// X[x0 + i, c] (+/-)= sum_k A[i + k*lda] * B[k + c*kT] straight into global X with
// atomics (i < m, c < nr, k < kk); A column-major with leading dimension lda.  With
// rows, output i goes to X row x0 + rows[i] instead.
template <bool kTrans>
__device__ __forceinline__ void block_gemv_atomic(double* X, int64_t ldx, int x0, const double* A, int lda,
                                                  const double* B, int m, int kk, int nr, double sign,
                                                  const int32_t* rows = nullptr) {
  if (m * nr * 4 <= kThreads) {  // few outputs (one or two right-hand sides): 4 threads per output
    const int idx = threadIdx.x >> 2, part = threadIdx.x & 3;
    const int c = idx / max(m, 1), i = idx - c * m;
    double s = 0.0;
    if (idx < m * nr) {
      if (kTrans)
        for (int k = part; k < kk; k += 4) s = fma(A[k + i * lda], B[k + c * kT], s);
      else
        for (int k = part; k < kk; k += 4) s = fma(A[i + k * lda], B[k + c * kT], s);
    }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if (idx < m * nr && part == 0) atomicAdd(X + x0 + (rows ? rows[i] : i) + c * ldx, sign * s);
    return;
  }
  for (int idx = threadIdx.x; idx < m * nr; idx += kThreads) {
    int c = idx / m, i = idx - c * m;
    double s = 0.0;
    if (kTrans)
      for (int k = 0; k < kk; ++k) s = fma(A[k + i * lda], B[k + c * kT], s);
    else
      for (int k = 0; k < kk; ++k) s = fma(A[i + k * lda], B[k + c * kT], s);
    atomicAdd(X + x0 + (rows ? rows[i] : i) + c * ldx, sign * s);
  }
}

// Lower-triangular solves of a kk x kk block held in A (ld lda) against the
// right-hand sides acc (ld kT), one warp per right-hand side column; rinv holds
// the reciprocals of the diagonal (computed off the dependency chain).
// forward: acc <- D^-1 acc ; backward: acc <- D^-T acc.
template <bool kForward>
__device__ void block_trsv(double* acc, const double* A, const double* rinv, int kk, int nr, int lda = kPld) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = kThreads / 32;
  for (int c = warp; c < nr; c += nw) {
    double v0 = lane < kk ? acc[lane + c * kT] : 0.0;
    double v1 = lane + 32 < kk ? acc[lane + 32 + c * kT] : 0.0;
    for (int step = 0; step < kk; ++step) {
      const int k = kForward ? step : kk - 1 - step;
      const int owner = k & 31;
      const bool hi = k >= 32;
      double xk = __shfl_sync(0xffffffffu, hi ? v1 : v0, owner) * rinv[k];
      if (lane == owner) {
        if (hi) v1 = xk;
        else v0 = xk;
      }
      if (kForward) {
        // rows j > k: acc_j -= D[j][k] x_k
        if (lane > k && lane < kk) v0 = fma(-A[lane + k * lda], xk, v0);
        if (lane + 32 > k && lane + 32 < kk) v1 = fma(-A[lane + 32 + k * lda], xk, v1);
      } else {
        // rows j < k: acc_j -= D[k][j] x_k
        if (lane < k) v0 = fma(-A[k + lane * lda], xk, v0);
        if (lane + 32 < k) v1 = fma(-A[k + (lane + 32) * lda], xk, v1);
      }
    }
    if (lane < kk) acc[lane + c * kT] = v0;
    if (lane + 32 < kk) acc[lane + 32 + c * kT] = v1;
  }
}

// Inverses of the eight 8 x 8 diagonal blocks of a full 64 x 64 lower block A (ld kPld),
// written transposed into A's unused upper triangle: Inv_g[i][j] (i > j) at
// A[(8g + j) + (8g + i) * kPld]; their diagonal is rinv.  Warp g inverts block g, lane j
// its column j by substitution.  Computed before a chain task waits, off the chain.
__device__ void invert_diag8(double* A, const double* rinv) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp >= 8 || lane >= 8) return;
  const int b = 8 * warp, j = lane;
  double z[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < i; ++k)
      if (k >= j) t = fma(A[(b + i) + (b + k) * kPld], z[k], t);
    z[i] = i < j ? 0.0 : (i == j ? rinv[b + i] : -t * rinv[b + i]);
  }
#pragma unroll
  for (int i = 1; i < 8; ++i)
    if (i > j) A[(b + j) + (b + i) * kPld] = z[i];
}

// block_trsv for a full 64 x 64 block whose 8 x 8 diagonal inverses invert_diag8 stored:
// eight groups of 8 rows, each solved by a product with its inverse (every lane computes
// the group's 8 values from 8 shuffled inputs) and applied to the rows not yet solved.
// forward: acc <- L^-1 acc ; backward: acc <- L^-T acc.  One warp per right-hand side.
template <bool kForward>
__device__ void block_trsv64(double* acc, const double* A, const double* rinv, int nr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = kThreads / 32;
  for (int c = warp; c < nr; c += nw) {
    double v0 = acc[lane + c * kT], v1 = acc[lane + 32 + c * kT];
#pragma unroll
    for (int step = 0; step < 8; ++step) {
      const int g = kForward ? step : 7 - step, b = 8 * g;
      const bool hi = g >= 4;  // the group's rows are held in v1 of lanes b - 32 ..
      double r[8], x[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) r[j] = __shfl_sync(0xffffffffu, hi ? v1 : v0, (b & 31) + j);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        double t = rinv[b + j] * r[j];
        if (kForward) {
#pragma unroll
          for (int m = 0; m < j; ++m) t = fma(A[(b + m) + (b + j) * kPld], r[m], t);  // Inv[j][m]
        } else {
#pragma unroll
          for (int m = j + 1; m < 8; ++m) t = fma(A[(b + j) + (b + m) * kPld], r[m], t);  // Inv[m][j]
        }
        x[j] = t;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (!hi && lane == b + j) v0 = x[j];
        if (hi && lane + 32 == b + j) v1 = x[j];
      }
      if (kForward) {  // rows below the group: v_r -= sum_j L[r][b + j] x_j
        if (lane > b + 7) {
#pragma unroll
          for (int j = 0; j < 8; ++j) v0 = fma(-A[lane + (b + j) * kPld], x[j], v0);
        }
        if (lane + 32 > b + 7) {
#pragma unroll
          for (int j = 0; j < 8; ++j) v1 = fma(-A[lane + 32 + (b + j) * kPld], x[j], v1);
        }
      } else {  // rows above the group: v_k -= sum_j L[b + j][k] x_j
        if (lane < b) {
#pragma unroll
          for (int j = 0; j < 8; ++j) v0 = fma(-A[(b + j) + lane * kPld], x[j], v0);
        }
        if (lane + 32 < b) {
#pragma unroll
          for (int j = 0; j < 8; ++j) v1 = fma(-A[(b + j) + (lane + 32) * kPld], x[j], v1);
        }
      }
    }
    acc[lane + c * kT] = v0;
    acc[lane + 32 + c * kT] = v1;
  }
}

// Next task of a persistent sweep; the whole block takes the same branch
// (thread 0 alone reads the counter and the status word, a barrier reached by
// only part of a block would hang).  -1 = no task left or a failure recorded.
__device__ __forceinline__ int next_task(const PSolveArgs& a, int* sh_task, int* sh_stop) {
  if (threadIdx.x == 0) {
    *sh_task = atomicAdd(a.counter, 1);
    *sh_stop = status_code(a.status) != 0;
  }
  __syncthreads();
  const int tk = *sh_task;
  const bool stop = *sh_stop != 0;
  __syncthreads();
  return (tk >= a.ntasks || stop) ? -1 : tk;
}

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Task timeline for analysis (thread 0; trace may be null).
__device__ __forceinline__ void trace_mark(const PSolveArgs& a, int tk, int slot, unsigned long long v) {
  if (a.trace && threadIdx.x == 0) a.trace[4 * (size_t)tk + slot] = v;
}

// Publish a block's writes, then bump a counter (thread 0).
__device__ __forceinline__ void signal(int32_t* counter) {
  __syncthreads();
  if (threadIdx.x == 0) red_release(counter, 1);
}

// Forward arrivals of one off-diagonal tile (panel rows r0 .. r1-1 of supernode s):
// one per target supernode, i.e. per relative-index group the rows span (groups are
// maximal runs of rows with the same target, numbered in row order), signalled in
// parallel after the block's scatter.
__device__ __forceinline__ void signal_arrivals(const PSolveArgs& a, const SnMeta& m, int r0, int r1) {
  __syncthreads();
  const int g0 = a.row_group[m.lidx + r0], g1 = a.row_group[m.lidx + r1 - 1];
  for (int g = g0 + (int)threadIdx.x; g <= g1; g += kThreads) red_release(a.arrived + a.groups[g].t, 1);
}

// Shape of super-block p of a supernode of nblk 64-column blocks.
struct SuperBlock {
  int b0, nb;  // first block, blocks
  __device__ SuperBlock(int p, int sb, int nblk) : b0(p * sb), nb(min(sb, nblk - p * sb)) {}
};

// First element of tile (r, q) (r >= q) of the inverse of super-block p.
template <class T>
__device__ __forceinline__ const T* inv_tile(const PSolveArgs& a, const SnMeta& m, int p, int r, int q) {
  const int64_t full = (int64_t)a.sb * (a.sb + 1) / 2;
  return static_cast<const T*>(a.Inv) + m.ioff + ((int64_t)p * full + (int64_t)r * (r + 1) / 2 + q) * (kT * kT);
}

// acc (64 x nr, ld kT) = sum_{j0 <= j < j1} tile_j (x) x_j, with the tile loads one
// ahead in registers (the caller has issued tile j0's).  tile(j, regs) issues the
// loads of tile j; xrow(j) gives the first X row of x_j, xlen(j) its valid rows;
// kTrans applies the tiles transposed; m = valid outputs.  The x blocks are staged
// all at once when they fit Bx.
template <class T, bool kTrans, class TileFn, class XRow, class XLen>
__device__ __forceinline__ void slab_product(double* acc, double* Ab, double* Bx, int j0, int j1, TileRegs<T>& regs,
                                             TileFn tile, const double* X, int64_t ldx, XRow xrow, XLen xlen,
                                             int m, int nr) {
  const int nt = j1 - j0;
  for (int idx = threadIdx.x; idx < kT * nr; idx += kThreads) acc[idx] = 0.0;
  const bool all = nt * kT * nr <= kT * kT;
  if (all)
    for (int j = 0; j < nt; ++j) stage_x(Bx + j * kT, nt * kT, X, ldx, xrow(j0 + j), nullptr, xlen(j0 + j), nr);
  for (int j = 0; j < nt; ++j) {
    regs.store(Ab);
    if (j + 1 < nt) tile(j0 + j + 1, regs);
    if (!all) stage_x(Bx, kT, X, ldx, xrow(j0 + j), nullptr, xlen(j0 + j), nr);
    __syncthreads();
    if (all) tile_gemv<kTrans>(acc, Ab, Bx + j * kT, nt * kT, m, xlen(j0 + j), nr);
    else tile_gemv<kTrans>(acc, Ab, Bx, kT, m, xlen(j0 + j), nr);
    __syncthreads();
  }
}

// out[x0 + i + c*ldx] += sign * acc[i + c*kT] for i < m, c < nr (atomic).
__device__ __forceinline__ void add_out(double* out, int64_t ldx, int x0, const double* acc, int m, int nr,
                                        double sign, const int32_t* rows = nullptr) {
  for (int idx = threadIdx.x; idx < m * nr; idx += kThreads) {
    int c = idx / m, i = idx - c * m;
    atomicAdd(out + x0 + (rows ? rows[i] : i) + c * ldx, sign * acc[i + c * kT]);
  }
}

// Forward sweep of one tiny leaf supernode s (w <= kTinyMaxW columns, no arrivals to wait
// for) by one thread: Z_0 <- L_00^-1 Y_0 by substitution (multiplying by the pivots'
// reciprocals), then Y[ancestor rows] -= L_u0 Z_0 with atomic additions, then one arrival
// per target group of its rows (the release orders the thread's own writes) and its
// diagonal-done count.
template <class T>
__device__ void tiny_forward(const PSolveArgs& a, int s, int nr) {
  const SnMeta m = a.meta[s];
  const T* P = static_cast<const T*>(a.L) + m.off;
  const int32_t* rl = a.rows + m.lidx;
  const int w = m.w, h = m.h;
  const int64_t ld = m.ld;
  double rinv[kTinyMaxW];
#pragma unroll
  for (int j = 0; j < kTinyMaxW; ++j) rinv[j] = j < w ? 1.0 / (double)P[j + j * ld] : 0.0;
  for (int c = 0; c < nr; ++c) {
    const int64_t xo = (int64_t)c * a.ldx;
    double y[kTinyMaxW];
#pragma unroll
    for (int j = 0; j < kTinyMaxW; ++j) {
      if (j >= w) break;
      double t = a.X[m.fc + j + xo];
#pragma unroll
      for (int k = 0; k < j; ++k) t = fma(-(double)P[j + k * ld], y[k], t);
      y[j] = t * rinv[j];
      a.Z[m.fc + j + xo] = y[j];
    }
    for (int r = w; r < h; ++r) {
      double t = 0.0;
#pragma unroll
      for (int j = 0; j < kTinyMaxW; ++j)
        if (j < w) t = fma((double)P[r + j * ld], y[j], t);
      atomicAdd(a.X + rl[r] + xo, -t);
    }
  }
  if (h > w) {
    const int g0 = a.row_group[m.lidx + w], g1 = a.row_group[m.lidx + h - 1];
    for (int g = g0; g <= g1; ++g) red_release(a.arrived + a.groups[g].t, 1);
  }
  red_release(a.blkdone + s, 1);
}

// Backward sweep of one tiny leaf supernode s by one thread, once its parent is done
// (bounded wait, like wait_geq but per thread): Z_0 -= L_u0^T X[ancestor rows], then
// X_0 <- L_00^-T Z_0 by substitution; then its diagonal-done count.
template <class T>
__device__ void tiny_backward(const PSolveArgs& a, int s, int nr) {
  const SnMeta m = a.meta[s];
  const int par = a.sparent[s];
  if (par >= 0) {
    const int target = solve_done_count(a.meta[par].w, a.sb, a.tpt);
    const int32_t* flag = a.blkdone + par;
    if (ld_acquire(flag) < target) {
      bool good = false;
      for (long long it = 0; it < a.spin_limit; ++it) {
        if (it >= 256) __nanosleep(128);
        if (ld_acquire(flag) >= target) {
          good = true;
          break;
        }
        if (status_code(a.status) != 0) return;
      }
      if (!good) {
        report_status(a.status, 3, s, target);
        return;
      }
    }
  }
  const T* P = static_cast<const T*>(a.L) + m.off;
  const int32_t* rl = a.rows + m.lidx;
  const int w = m.w, h = m.h;
  const int64_t ld = m.ld;
  double rinv[kTinyMaxW];
#pragma unroll
  for (int j = 0; j < kTinyMaxW; ++j) rinv[j] = j < w ? 1.0 / (double)P[j + j * ld] : 0.0;
  for (int c = 0; c < nr; ++c) {
    const int64_t xo = (int64_t)c * a.ldx;
    double z[kTinyMaxW];
#pragma unroll
    for (int j = 0; j < kTinyMaxW; ++j) z[j] = j < w ? a.Z[m.fc + j + xo] : 0.0;
    for (int r = w; r < h; ++r) {
      const double xr = a.X[rl[r] + xo];
#pragma unroll
      for (int j = 0; j < kTinyMaxW; ++j)
        if (j < w) z[j] = fma(-(double)P[r + j * ld], xr, z[j]);
    }
#pragma unroll
    for (int j = kTinyMaxW - 1; j >= 0; --j) {
      if (j >= w) continue;
      double t = z[j];
#pragma unroll
      for (int k = j + 1; k < kTinyMaxW; ++k)
        if (k < w) t = fma(-(double)P[k + j * ld], z[k], t);
      z[j] = t * rinv[j];
      a.X[m.fc + j + xo] = z[j];
    }
  }
  red_release(a.blkdone + s, 1);
}

template <class T, int kR>
__global__ void __launch_bounds__(kThreads, solve_min_blocks<kR>()) k_solve_forward(PSolveArgs a) {
  extern __shared__ __align__(16) double sm[];
  double* Ab = sm;                  // staged tile, ld kPld
  double* Bx = sm + kT * kPld;      // staged right-hand-side rows
  double* acc = Bx + kT * kT;       // accumulator, ld kT
  __shared__ int sh_task, sh_stop, sh_ok;
  __shared__ double sh_rinv[kT];
  const int nr = a.nrhs;
  TileRegs<T> regs;
  for (;;) {
    const int tk = next_task(a, &sh_task, &sh_stop);
    if (tk < 0) return;
    const SolveTask task = a.tasks[tk];
    const int s = task.s;
    trace_mark(a, tk, 0, now_ns());
    trace_mark(a, tk, 3, ((unsigned long long)s << 8) | (unsigned)task.kind);
    const SnMeta m = a.meta[s];
    const T* P = static_cast<const T*>(a.L) + m.off;
    const int32_t* rl = a.rows + m.lidx;
    const int64_t ld = m.ld;
    const int nblk = (m.w + kT - 1) / kT;
    if (task.kind == 6) {
      // T: tiny leaf supernodes, one per thread (nothing to wait for)
      trace_mark(a, tk, 1, now_ns());
      if ((int)threadIdx.x < task.t) tiny_forward<T>(a, a.tiny[task.i + threadIdx.x], nr);
      __syncthreads();
    } else if (task.kind == 5) {
      // DI(p, r): Z[block r of p] += sum_{q <= r, this task's tiles} Inv_p(r, q) Y[block q of p]
      const int p = task.i & 0xffffff, q0 = task.i >> 24, r = task.t;
      const SuperBlock B(p, a.sb, nblk);
      const int t = B.b0 + r, bt = min(kT, m.w - t * kT), q1 = min(r + 1, q0 + a.tpt);
      auto tile = [&](int q, TileRegs<T>& R) { R.load(inv_tile<T>(a, m, p, r, q), kT, kT, kT); };
      tile(q0, regs);  // the inverse is final: load before waiting
      if (!wait_geq(a.arrived + s, a.expected[s], a.status, s, &sh_ok, a.spin_limit)) return;
      if (!wait_geq(a.upd + m.sboff + p, p * B.nb * solve_ntask(a.sb, a.tpt), a.status, s, &sh_ok, a.spin_limit))
        return;
      trace_mark(a, tk, 1, now_ns());
      slab_product<T, false>(
          acc, Ab, Bx, q0, q1, regs, tile, a.X, a.ldx, [&](int q) { return m.fc + (B.b0 + q) * kT; },
          [&](int q) { return min(kT, m.w - (B.b0 + q) * kT); }, bt, nr);
      add_out(a.Z, a.ldx, m.fc + t * kT, acc, bt, nr, 1.0);
      signal(a.blkdone + s);
    } else if (task.kind == 1) {
      // U(p, t): Y[block t] -= L(t, super-block p) Z[p] over this task's tiles
      const int p = task.i & 0xffffff, q0 = task.i >> 24, t = task.t;
      const SuperBlock B(p, a.sb, nblk);
      const int r0 = t * kT, bt = min(kT, m.w - r0), q1 = min(B.nb, q0 + a.tpt);
      auto tile = [&](int q, TileRegs<T>& R) {
        const int c0 = (B.b0 + q) * kT;
        R.load(P + r0 + (int64_t)c0 * ld, ld, bt, min(kT, m.w - c0));
      };
      tile(q0, regs);  // L is final: load before waiting
      if (!wait_geq(a.blkdone + s, solve_di_range(nblk, a.sb, a.tpt, 0, p + 1), a.status, s, &sh_ok, a.spin_limit))
        return;
      trace_mark(a, tk, 1, now_ns());
      slab_product<T, false>(
          acc, Ab, Bx, q0, q1, regs, tile, a.Z, a.ldx, [&](int q) { return m.fc + (B.b0 + q) * kT; },
          [&](int q) { return min(kT, m.w - (B.b0 + q) * kT); }, bt, nr);
      add_out(a.X, a.ldx, m.fc + r0, acc, bt, nr, -1.0);
      signal(a.upd + m.sboff + t / a.sb);
    } else if (task.kind == 2) {
      // O(p, u): Y[ancestor rows of tile u] -= L(u, super-block p) Z[p] over this task's tiles
      const int p = task.i & 0xffffff, q0 = task.i >> 24, u = task.t, r0 = m.w + u * kT, bu = min(kT, m.h - r0);
      const SuperBlock B(p, a.sb, nblk);
      const int q1 = min(B.nb, q0 + a.tpt);
      auto tile = [&](int q, TileRegs<T>& R) {
        const int c0 = (B.b0 + q) * kT;
        R.load(P + r0 + (int64_t)c0 * ld, ld, bu, min(kT, m.w - c0));
      };
      tile(q0, regs);
      if (!wait_geq(a.blkdone + s, solve_di_range(nblk, a.sb, a.tpt, 0, p + 1), a.status, s, &sh_ok, a.spin_limit))
        return;
      trace_mark(a, tk, 1, now_ns());
      slab_product<T, false>(
          acc, Ab, Bx, q0, q1, regs, tile, a.Z, a.ldx, [&](int q) { return m.fc + (B.b0 + q) * kT; },
          [&](int q) { return min(kT, m.w - (B.b0 + q) * kT); }, bu, nr);
      add_out(a.X, a.ldx, 0, acc, bu, nr, -1.0, rl + r0);
      signal_arrivals(a, m, r0, r0 + bu);
      __syncthreads();
    } else if (task.kind == 0) {
      // D: one-block supernode, Z_0 <- L_00^-1 Y_0 (its off-diagonal tiles are O tasks)
      const int w = m.w;
      stage_block(Ab, P, ld, 0, w, 0, w);  // L is final: load before waiting
      __syncthreads();
      if (threadIdx.x < w) sh_rinv[threadIdx.x] = 1.0 / Ab[threadIdx.x * (kPld + 1)];
      if (w == kT) {  // full block: 8 x 8 diagonal inverses, off the chain
        __syncthreads();
        invert_diag8(Ab, sh_rinv);
      }
      if (!wait_geq(a.arrived + s, a.expected[s], a.status, s, &sh_ok, a.spin_limit)) return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(acc, kT, a.X, a.ldx, m.fc, nullptr, w, nr);
      __syncthreads();
      if (w == kT) block_trsv64<true>(acc, Ab, sh_rinv, nr);
      else block_trsv<true>(acc, Ab, sh_rinv, w, nr);
      __syncthreads();
      for (int idx = threadIdx.x; idx < w * nr; idx += kThreads) {
        int c = idx / w, i = idx - c * w;
        a.Z[m.fc + i + c * a.ldx] = acc[i + c * kT];
      }
      signal(a.blkdone + s);
    } else {
      // F: one-block supernode whole: Z_0 <- L_00^-1 Y_0, then every off-diagonal tile's
      // Y[ancestor rows] -= L_u0 Z_0
      const int w = m.w, h = m.h, noff = (m.h - m.w + kT - 1) / kT;
      // a panel that fits the two staging buffers is loaded whole (ld h) before waiting
      const bool whole = h * w <= kT * kPld + kT * kT;
      if (whole) {  // eight loads of a thread in flight at a time
        for (int base = threadIdx.x; base < h * w; base += 8 * kThreads) {
          T v[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int idx = base + q * kThreads, c = idx / h, r = idx - c * h;
            v[q] = idx < h * w ? P[r + (int64_t)c * ld] : T(0);
          }
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (base + q * kThreads < h * w) Ab[base + q * kThreads] = (double)v[q];
        }
      } else {
        stage_block(Ab, P, ld, 0, w, 0, w);  // L is final: load before waiting
      }
      const int lda = whole ? h : kPld;
      __syncthreads();
      if (threadIdx.x < w) sh_rinv[threadIdx.x] = 1.0 / Ab[threadIdx.x * (lda + 1)];
      if (!wait_geq(a.arrived + s, a.expected[s], a.status, s, &sh_ok, a.spin_limit)) return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(acc, kT, a.X, a.ldx, m.fc, nullptr, w, nr);
      __syncthreads();
      block_trsv<true>(acc, Ab, sh_rinv, w, nr, lda);
      __syncthreads();
      for (int idx = threadIdx.x; idx < w * nr; idx += kThreads) {
        int c = idx / w, i = idx - c * w;
        a.Z[m.fc + i + c * a.ldx] = acc[i + c * kT];
      }
      for (int u = 0; u < noff; ++u) {
        const int r0 = w + u * kT, bu = min(kT, m.h - r0);
        if (!whole) {
          stage_block(Ab, P, ld, r0, bu, 0, w);
          __syncthreads();
        }
        block_gemv_atomic<false>(a.X, a.ldx, 0, whole ? Ab + r0 : Ab, lda, acc, bu, w, nr, -1.0, rl + r0);
        signal_arrivals(a, m, r0, r0 + bu);  // one per (tile, target), as the plan counts them
        __syncthreads();
      }
      if (threadIdx.x == 0) red_release(a.blkdone + s, 1);
    }
    trace_mark(a, tk, 2, now_ns());
  }
}

template <class T, int kR>
__global__ void __launch_bounds__(kThreads, solve_min_blocks<kR>()) k_solve_backward(PSolveArgs a) {
  extern __shared__ __align__(16) double sm[];
  double* Ab = sm;
  double* Bx = sm + kT * kPld;
  double* acc = Bx + kT * kT;
  __shared__ int sh_task, sh_stop, sh_ok;
  __shared__ double sh_rinv[kT];
  const int nr = a.nrhs;
  TileRegs<T> regs;
  for (;;) {
    const int tk = next_task(a, &sh_task, &sh_stop);
    if (tk < 0) return;
    const SolveTask task = a.tasks[tk];
    const int s = task.s;
    trace_mark(a, tk, 0, now_ns());
    trace_mark(a, tk, 3, ((unsigned long long)s << 8) | (unsigned)task.kind);
    const SnMeta m = a.meta[s];
    const T* P = static_cast<const T*>(a.L) + m.off;
    const int32_t* rl = a.rows + m.lidx;
    const int64_t ld = m.ld;
    const int nblk = (m.w + kT - 1) / kT, nsb = (nblk + a.sb - 1) / a.sb;
    const int noff = (m.h - m.w + kT - 1) / kT;
    if (task.kind == 6) {
      // T: tiny leaf supernodes, one per thread (each waits for its parent)
      trace_mark(a, tk, 1, now_ns());
      if ((int)threadIdx.x < task.t) tiny_backward<T>(a, a.tiny[task.i + threadIdx.x], nr);
      __syncthreads();
      if (status_code(a.status) != 0) return;
    } else if (task.kind == 5) {
      // DI(p, r): X[block r of p] += sum_{q >= r, this task's tiles} Inv_p(q, r)^T Z[block q of p]
      const int p = task.i & 0xffffff, j0 = task.i >> 24, r = task.t;
      const SuperBlock B(p, a.sb, nblk);
      const int t = B.b0 + r, bt = min(kT, m.w - t * kT), j1 = min(B.nb - r, j0 + a.tpt);
      auto tile = [&](int j, TileRegs<T>& R) { R.load(inv_tile<T>(a, m, p, r + j, r), kT, kT, kT); };
      tile(j0, regs);
      // W tasks of every off-diagonal tile, V tasks of every later super-block into each block of p
      const int nlast = nblk - (nsb - 1) * a.sb;
      const int later = p < nsb - 1 ? (nsb - 2 - p) * solve_ntask(a.sb, a.tpt) + solve_ntask(nlast, a.tpt) : 0;
      if (!wait_geq(a.upd + m.sboff + p, noff * solve_ntask(B.nb, a.tpt) + B.nb * later, a.status, s, &sh_ok,
                    a.spin_limit))
        return;
      trace_mark(a, tk, 1, now_ns());
      slab_product<T, true>(
          acc, Ab, Bx, j0, j1, regs, tile, a.Z, a.ldx, [&](int j) { return m.fc + (t + j) * kT; },
          [&](int j) { return min(kT, m.w - (t + j) * kT); }, bt, nr);
      add_out(a.X, a.ldx, m.fc + t * kT, acc, bt, nr, 1.0);
      signal(a.blkdone + s);
    } else if (task.kind == 1) {
      // V(p, t): Z[block t] -= L(super-block p, t)^T X[p] over this task's tiles
      const int p = task.i & 0xffffff, q0 = task.i >> 24, t = task.t, c0 = t * kT, bt = min(kT, m.w - c0);
      const SuperBlock B(p, a.sb, nblk);
      const int q1 = min(B.nb, q0 + a.tpt);
      auto tile = [&](int q, TileRegs<T>& R) {
        const int r0 = (B.b0 + q) * kT;
        R.load(P + r0 + (int64_t)c0 * ld, ld, min(kT, m.w - r0), bt);
      };
      tile(q0, regs);
      if (!wait_geq(a.blkdone + s, solve_di_range(nblk, a.sb, a.tpt, p, nsb), a.status, s, &sh_ok, a.spin_limit))
        return;
      trace_mark(a, tk, 1, now_ns());
      slab_product<T, true>(
          acc, Ab, Bx, q0, q1, regs, tile, a.X, a.ldx, [&](int q) { return m.fc + (B.b0 + q) * kT; },
          [&](int q) { return min(kT, m.w - (B.b0 + q) * kT); }, bt, nr);
      add_out(a.Z, a.ldx, m.fc + c0, acc, bt, nr, -1.0);
      signal(a.upd + m.sboff + t / a.sb);
    } else if (task.kind == 3) {
      // W(p, u): Z[p] -= L(u, super-block p)^T X[ancestor rows of tile u] over this task's
      // tiles, final once the parent is done
      const int p = task.i & 0xffffff, q0 = task.i >> 24, u = task.t, rr = m.w + u * kT, br = min(kT, m.h - rr);
      const SuperBlock B(p, a.sb, nblk);
      const int q1 = min(B.nb, q0 + a.tpt);
      const int par = a.sparent[s];
      regs.load(P + rr + (int64_t)(B.b0 + q0) * kT * ld, ld, br, min(kT, m.w - (B.b0 + q0) * kT));
      if (par >= 0 &&
          !wait_geq(a.blkdone + par, solve_done_count(a.meta[par].w, a.sb, a.tpt), a.status, s, &sh_ok, a.spin_limit))
        return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(Bx, kT, a.X, a.ldx, 0, rl + rr, br, nr);
      for (int q = q0; q < q1; ++q) {
        const int c0 = (B.b0 + q) * kT, bq = min(kT, m.w - c0);
        regs.store(Ab);
        if (q + 1 < q1) {
          const int c1 = c0 + kT;
          regs.load(P + rr + (int64_t)c1 * ld, ld, br, min(kT, m.w - c1));
        }
        __syncthreads();
        block_gemv_atomic<true>(a.Z, a.ldx, m.fc + c0, Ab, kPld, Bx, bq, br, nr, -1.0);
        __syncthreads();
      }
      if (threadIdx.x == 0) red_release(a.upd + m.sboff + p, 1);
    } else if (task.kind == 0) {
      // B: one-block supernode, X_0 <- L_00^-T Z_0 once its W updates landed
      const int w = m.w;
      stage_block(Ab, P, ld, 0, w, 0, w);  // L is final: load before waiting
      __syncthreads();
      if (threadIdx.x < w) sh_rinv[threadIdx.x] = 1.0 / Ab[threadIdx.x * (kPld + 1)];
      if (w == kT) {  // full block: 8 x 8 diagonal inverses, off the chain
        __syncthreads();
        invert_diag8(Ab, sh_rinv);
      }
      if (!wait_geq(a.upd + m.sboff, noff, a.status, s, &sh_ok, a.spin_limit)) return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(acc, kT, a.Z, a.ldx, m.fc, nullptr, w, nr);
      __syncthreads();
      if (w == kT) block_trsv64<false>(acc, Ab, sh_rinv, nr);
      else block_trsv<false>(acc, Ab, sh_rinv, w, nr);
      __syncthreads();
      for (int idx = threadIdx.x; idx < w * nr; idx += kThreads) {
        int c = idx / w, i = idx - c * w;
        a.X[m.fc + i + c * a.ldx] = acc[i + c * kT];
      }
      signal(a.blkdone + s);
    } else {
      // G: one-block supernode whole: Z_0 -= L_u0^T X_u for every off-diagonal tile
      // (ancestor rows, final once the parent is done), then X_0 <- L_00^-T Z_0
      const int w = m.w;
      const int par = a.sparent[s];
      if (par >= 0 &&
          !wait_geq(a.blkdone + par, solve_done_count(a.meta[par].w, a.sb, a.tpt), a.status, s, &sh_ok, a.spin_limit))
        return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(acc, kT, a.Z, a.ldx, m.fc, nullptr, w, nr);
      for (int u = 0; u < noff; ++u) {
        const int r0 = w + u * kT, bu = min(kT, m.h - r0);
        __syncthreads();
        stage_block(Ab, P, ld, r0, bu, 0, w);
        stage_x(Bx, kT, a.X, a.ldx, 0, rl + r0, bu, nr);
        __syncthreads();
        for (int idx = threadIdx.x; idx < w * nr; idx += kThreads) {  // acc_k -= sum_r L_rk x_r
          const int c = idx / w, k = idx - c * w;
          double t = 0.0;
          for (int r = 0; r < bu; ++r) t = fma(Ab[r + k * kPld], Bx[r + c * kT], t);
          acc[k + c * kT] -= t;
        }
      }
      __syncthreads();
      stage_block(Ab, P, ld, 0, w, 0, w);
      __syncthreads();
      if (threadIdx.x < w) sh_rinv[threadIdx.x] = 1.0 / Ab[threadIdx.x * (kPld + 1)];
      __syncthreads();
      block_trsv<false>(acc, Ab, sh_rinv, w, nr);
      __syncthreads();
      for (int idx = threadIdx.x; idx < w * nr; idx += kThreads) {
        int c = idx / w, i = idx - c * w;
        a.X[m.fc + i + c * a.ldx] = acc[i + c * kT];
      }
      __syncthreads();
      if (threadIdx.x == 0) red_release(a.blkdone + s, 1);
    }
    trace_mark(a, tk, 2, now_ns());
  }
}

// ---- diagonal super-block inverses ---------------------------------------------------
// One CTA per (super-block p, column block j): the tiles Inv(i, j), i = j .. nb - 1, of
// Inv_p = L_pp^-1 by block substitution down column j:
//   Inv(j, j) = L_jj^-1,   Inv(i, j) = -L_ii^-1 sum_{k=j}^{i-1} L_ik Inv(k, j),
// in FP64 (the panel widened), stored in the arena's type.  The tiles of column j above
// tile i are this CTA's own earlier writes, read back through L2.
constexpr int kInvThreads = 256;
constexpr size_t kInvSmem = (size_t)3 * kT * kPld * sizeof(double);  // two CTAs per SM

// C (64 x 64, ld kPld) = A * B or += A * B (both 64 x 64, ld kPld); thread (ty, tx)
// owns C[ty + 16 ii][tx + 16 jj].
template <bool kAccumulate>
__device__ __forceinline__ void gemm64(double* C, const double* A, const double* B, double scale) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double c[4][4] = {};
  for (int k = 0; k < kT; ++k) {
    double av[4], bv[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) av[i] = A[ty + 16 * i + k * kPld];
#pragma unroll
    for (int j = 0; j < 4; ++j) bv[j] = B[k + (tx + 16 * j) * kPld];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) c[i][j] = fma(av[i], bv[j], c[i][j]);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      double& d = C[ty + 16 * i + (tx + 16 * j) * kPld];
      d = kAccumulate ? d + scale * c[i][j] : scale * c[i][j];
    }
}

// Ti = inverse of the b x b lower triangle of Ls (both ld kPld; zero outside b x b).
// Four threads per column c: x_i = (delta_ic - sum_{k<i} L_ik x_k) / L_ii down the column.
__device__ __forceinline__ void tri_inverse64(double* Ti, const double* Ls, int b) {
  const int c = threadIdx.x >> 2, part = threadIdx.x & 3;
  for (int i = 0; i < kT; ++i) {
    double s = 0.0;
    if (i < b && c < b && i > c)
      for (int k = c + part; k < i; k += 4) s = fma(Ls[i + k * kPld], Ti[k + c * kPld], s);
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if (part == 0) {
      double x = 0.0;
      if (i < b && c < b && i >= c) x = (i == c ? 1.0 : -s) / Ls[i + i * kPld];
      Ti[i + c * kPld] = x;
    }
    __syncwarp();
  }
}

template <class T>
__global__ void __launch_bounds__(kInvThreads, 2) k_sb_inverse(const T* __restrict__ L, T* __restrict__ Inv,
                                                               const SnMeta* __restrict__ meta,
                                                               const InvItem* __restrict__ items, int sb) {
  extern __shared__ __align__(16) double smi[];
  double* Ls = smi;               // L(i, k), then L(i, i), then the output tile
  double* Ti = Ls + kT * kPld;    // Inv(k, j) while accumulating, then L(i, i)^-1
  double* Acc = Ti + kT * kPld;
  const InvItem it = items[blockIdx.x];
  const SnMeta m = meta[it.s];
  const int nblk = (m.w + kT - 1) / kT, b0 = it.p * sb, nb = min(sb, nblk - b0), j = it.j;
  const int64_t full = (int64_t)sb * (sb + 1) / 2;
  T* base = Inv + m.ioff + (int64_t)it.p * full * (kT * kT);
  const T* P = L + m.off;
  const int64_t ld = m.ld;
  auto tile_ptr = [&](int r, int q) { return base + ((int64_t)r * (r + 1) / 2 + q) * (kT * kT); };
  auto stage_L = [&](double* dst, int r0, int rb, int c0, int cb) {
    for (int idx = threadIdx.x; idx < kT * kT; idx += kInvThreads) {
      const int k = idx >> 6, r = idx & 63;
      dst[r + k * kPld] = (r < rb && k < cb) ? (double)P[r0 + r + (int64_t)(c0 + k) * ld] : 0.0;
    }
  };
  for (int i = j; i < nb; ++i) {
    const int ci = (b0 + i) * kT, bi = min(kT, m.w - ci);
    if (i > j) {  // Acc = sum_{k=j}^{i-1} L_ik Inv(k, j)
      for (int k = j; k < i; ++k) {
        const int ck = (b0 + k) * kT, bk = min(kT, m.w - ck);
        stage_L(Ls, ci, bi, ck, bk);
        const T* src = tile_ptr(k, j);
        for (int idx = threadIdx.x; idx < kT * kT; idx += kInvThreads) {
          const int kk = idx >> 6, r = idx & 63;
          Ti[r + kk * kPld] = (double)__ldcg(src + idx);
        }
        __syncthreads();
        if (k == j) gemm64<false>(Acc, Ls, Ti, 1.0);
        else gemm64<true>(Acc, Ls, Ti, 1.0);
        __syncthreads();
      }
    }
    stage_L(Ls, ci, bi, ci, bi);
    __syncthreads();
    tri_inverse64(Ti, Ls, bi);
    __syncthreads();
    const double* out = Ti;
    if (i > j) {  // Inv(i, j) = -L_ii^-1 Acc
      gemm64<false>(Ls, Ti, Acc, -1.0);
      __syncthreads();
      out = Ls;
    }
    T* dst = tile_ptr(i, j);
    for (int idx = threadIdx.x; idx < kT * kT; idx += kInvThreads) {
      const int kk = idx >> 6, r = idx & 63;
      dst[idx] = (T)out[r + kk * kPld];
    }
    __syncthreads();
  }
}

}  // namespace

int g_solve_grid = 0;    // CTAs of the persistent sweeps (resident CTAs of the device)
int g_solve_grid16 = 0;  // CTAs of the persistent sweeps for <= 16 right-hand sides

void init_solve_attributes() {
  for (auto f : {k_solve_forward<double, 64>, k_solve_backward<double, 64>, k_solve_forward<float, 64>,
                 k_solve_backward<float, 64>})
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem<64>());
  for (auto f : {k_solve_forward<double, 16>, k_solve_backward<double, 16>, k_solve_forward<float, 16>,
                 k_solve_backward<float, 16>})
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem<16>());
  cudaFuncSetAttribute(k_sb_inverse<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInvSmem);
  cudaFuncSetAttribute(k_sb_inverse<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInvSmem);
  int dev = 0, sms = 0, per = 0, per16 = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_solve_forward<double, 64>, kThreads, solve_smem<64>());
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per16, k_solve_forward<double, 16>, kThreads, solve_smem<16>());
  g_solve_grid = sms * (per > 0 ? per : 1);
  if (g_solve_grid <= 0) g_solve_grid = 148;
  g_solve_grid16 = sms * (per16 > 0 ? per16 : 1);
  if (g_solve_grid16 <= 0) g_solve_grid16 = g_solve_grid;
}

void launch_sb_inverse(cudaStream_t st, const void* L, void* Inv, bool fp32, const SnMeta* meta,
                       const InvItem* items, int count, int sb) {
  if (count <= 0) return;
  if (fp32)
    k_sb_inverse<float><<<count, kInvThreads, kInvSmem, st>>>(static_cast<const float*>(L), static_cast<float*>(Inv),
                                                              meta, items, sb);
  else
    k_sb_inverse<double><<<count, kInvThreads, kInvSmem, st>>>(static_cast<const double*>(L),
                                                               static_cast<double*>(Inv), meta, items, sb);
}

void launch_solve_persistent(cudaStream_t st, const PSolveArgs& a, bool forward) {
  if (a.ntasks <= 0 || a.spin_limit <= 0) return;
  const bool small = a.nrhs <= 16;
  const int cap = small ? g_solve_grid16 : g_solve_grid;
  const int grid = cap < a.ntasks ? cap : a.ntasks;
  if (small) {
    const size_t sm = solve_smem<16>();
    if (a.fp32) {
      if (forward) k_solve_forward<float, 16><<<grid, kThreads, sm, st>>>(a);
      else k_solve_backward<float, 16><<<grid, kThreads, sm, st>>>(a);
    } else {
      if (forward) k_solve_forward<double, 16><<<grid, kThreads, sm, st>>>(a);
      else k_solve_backward<double, 16><<<grid, kThreads, sm, st>>>(a);
    }
    return;
  }
  const size_t sm = solve_smem<64>();
  if (a.fp32) {
    if (forward) k_solve_forward<float, 64><<<grid, kThreads, sm, st>>>(a);
    else k_solve_backward<float, 64><<<grid, kThreads, sm, st>>>(a);
  } else {
    if (forward) k_solve_forward<double, 64><<<grid, kThreads, sm, st>>>(a);
    else k_solve_backward<double, 64><<<grid, kThreads, sm, st>>>(a);
  }
}

}  // namespace dev
}  // namespace spb
