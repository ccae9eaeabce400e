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
// synchronise through per-supernode counters in global memory.  Every wait is
// bounded; on expiry the kernel records SPB timeout status and all CTAs leave.
#include "kernels.cuh"

namespace spb {
namespace dev {

namespace {

constexpr int kT = 64;         // rows / columns per task unit
constexpr int kPld = 65;       // padded leading dimension of the staged L block
constexpr int kThreads = 256;
// staged L block (64 x 65), a second 64 x 64 block (X rows or the next L block), and
// the accumulator of kR right-hand sides; kR = 16 keeps three CTAs per SM
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

// Counter increment with release semantics: after a barrier, one thread's release
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

// acc[i + c*kT] (+/-)= sum_k A[i + k*kPld] * B[k + c*kT]   for i < m, c < nr, k < kk
template <bool kSub>
__device__ __forceinline__ void block_gemv(double* acc, const double* A, const double* B, int m, int kk, int nr) {
  for (int idx = threadIdx.x; idx < m * nr; idx += kThreads) {
    int c = idx / m, i = idx - c * m;
    double s = 0.0;
    for (int k = 0; k < kk; ++k) s = fma(A[i + k * kPld], B[k + c * kT], s);
    if (kSub) acc[i + c * kT] -= s;
    else acc[i + c * kT] += s;
  }
}

// Stage L rows [r0, r0+m) x columns [c0, c0+kk) of a panel into A (ld kPld), widened to FP64.
// A full 64 x 64 block is loaded with all 16 loads of a thread in flight.
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

// Stage X rows x0.. (contiguous) or rows rl[0..] (gathered) into B (ld kT), through L2.
__device__ __forceinline__ void stage_x(double* B, const double* X, int64_t ldx, int x0, const int32_t* rl, int m,
                                        int nr) {
  for (int idx = threadIdx.x; idx < m * nr; idx += kThreads) {
    int c = idx / m, r = idx - c * m;
    int row = rl ? rl[r] : x0 + r;
    B[r + c * kT] = __ldcg(X + row + c * ldx);
  }
}

}  // namespace

namespace {

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

// Lower-triangular solves of a kk x kk block held in A (ld kPld) against the
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

template <class T, int kR>
__global__ void __launch_bounds__(kThreads, solve_min_blocks<kR>()) k_solve_forward(PSolveArgs a) {
  extern __shared__ __align__(16) double sm[];
  double* Ab = sm;                  // staged L block, ld kPld
  double* Bx = sm + kT * kPld;      // staged X rows, ld kT
  double* acc = Bx + kT * kT;       // accumulator, ld kT
  __shared__ int sh_task, sh_stop, sh_ok;
  __shared__ double sh_rinv[kT];
  const int nr = a.nrhs;
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
    if (task.kind == 0) {
      // D(t): descendants' and earlier blocks' updates have landed in X_t; X_t <- L_tt^-1 X_t,
      // then the update of the next block, X_{t+1} -= L_{t+1,t} X_t
      const int t = task.t, r0 = t * kT, bt = min(kT, m.w - r0);
      const int r1 = r0 + kT, b1 = r1 < m.w ? min(kT, m.w - r1) : 0;
      stage_block(Ab, P, ld, r0, bt, r0, bt);  // L is final: load before waiting
      if (b1) stage_block<T, kT>(Bx, P, ld, r1, b1, r0, bt);
      __syncthreads();
      if (threadIdx.x < bt) sh_rinv[threadIdx.x] = 1.0 / Ab[threadIdx.x * (kPld + 1)];
      if (bt == kT) {  // full block: 8 x 8 diagonal inverses, off the chain
        __syncthreads();
        invert_diag8(Ab, sh_rinv);
      }
      if (!wait_geq(a.arrived + s, a.expected[s], a.status, s, &sh_ok, a.spin_limit)) return;
      if (!wait_geq(a.upd + m.boff + t, t, a.status, s, &sh_ok, a.spin_limit)) return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(acc, a.X, a.ldx, m.fc + r0, nullptr, bt, nr);
      __syncthreads();
      if (bt == kT) block_trsv64<true>(acc, Ab, sh_rinv, nr);
      else block_trsv<true>(acc, Ab, sh_rinv, bt, nr);
      __syncthreads();
      for (int idx = threadIdx.x; idx < bt * nr; idx += kThreads) {
        int c = idx / bt, r = idx - c * bt;
        a.X[m.fc + r0 + r + c * a.ldx] = acc[r + c * kT];
      }
      if (b1) block_gemv_atomic<false>(a.X, a.ldx, m.fc + r1, Bx, kT, acc, b1, bt, nr, -1.0);
      __syncthreads();
      if (threadIdx.x == 0) {
        if (b1) red_release(a.upd + m.boff + t + 1, 1);  // the next block first: it is on the chain
        red_release(a.blkdone + s, 1);
      }
    } else if (task.kind == 1) {
      // U(i, t): X_t -= L_ti X_i
      const int i = task.i, t = task.t, bi = min(kT, m.w - i * kT), r0 = t * kT, bt = min(kT, m.w - r0);
      stage_block(Ab, P, ld, r0, bt, i * kT, bi);  // L is final: load before waiting
      if (!wait_geq(a.blkdone + s, i + 1, a.status, s, &sh_ok, a.spin_limit)) return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(Bx, a.X, a.ldx, m.fc + i * kT, nullptr, bi, nr);
      for (int idx = threadIdx.x; idx < kT * nr; idx += kThreads) acc[idx] = 0.0;
      __syncthreads();
      block_gemv<false>(acc, Ab, Bx, bt, bi, nr);
      __syncthreads();
      for (int idx = threadIdx.x; idx < bt * nr; idx += kThreads) {
        int c = idx / bt, r = idx - c * bt;
        atomicAdd(a.X + m.fc + r0 + r + c * a.ldx, -acc[r + c * kT]);
      }
      signal(a.upd + m.boff + t);
    } else if (task.kind == 4) {
      // F: a one-block supernode whole: X_0 <- L_00^-1 X_0, then every off-diagonal tile
      // scattered into the ancestors' rows
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
      stage_x(acc, a.X, a.ldx, m.fc, nullptr, w, nr);
      __syncthreads();
      block_trsv<true>(acc, Ab, sh_rinv, w, nr, lda);
      __syncthreads();
      for (int idx = threadIdx.x; idx < w * nr; idx += kThreads) {
        int c = idx / w, r = idx - c * w;
        a.X[m.fc + r + c * a.ldx] = acc[r + c * kT];
      }
      for (int u = 0; u < noff; ++u) {
        const int r0 = w + u * kT, bu = min(kT, m.h - r0);
        if (!whole) {
          stage_block(Ab, P, ld, r0, bu, 0, w);
          __syncthreads();
        }
        block_gemv_atomic<false>(a.X, a.ldx, 0, whole ? Ab + r0 : Ab, lda, acc, bu, w, nr, -1.0, rl + r0);
        __syncthreads();
        if (threadIdx.x == 0) {
          __threadfence();
          int last = -1;
          for (int r = 0; r < bu; ++r) {
            int tgt = a.supmember[rl[r0 + r]];
            if (tgt != last) atomicAdd(a.arrived + tgt, 1);
            last = tgt;
          }
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) red_release(a.blkdone + s, 1);
    } else {
      // O(i0, u): off-diagonal rows, Y_K[rows] -= L_KJ Y_J over the column blocks of a
      // chunk, accumulated, then scattered into the ancestors' rows
      const int i0 = task.i, u = task.t, r0 = m.w + u * kT, bu = min(kT, m.h - r0);
      const int i1 = min((m.w + kT - 1) / kT, i0 + a.chunk);
      for (int idx = threadIdx.x; idx < kT * nr; idx += kThreads) acc[idx] = 0.0;
      for (int i = i0; i < i1; ++i) {
        const int bi = min(kT, m.w - i * kT);
        stage_block(Ab, P, ld, r0, bu, i * kT, bi);  // L is final: load before waiting
        if (!wait_geq(a.blkdone + s, i + 1, a.status, s, &sh_ok, a.spin_limit)) return;
        stage_x(Bx, a.X, a.ldx, m.fc + i * kT, nullptr, bi, nr);
        __syncthreads();
        block_gemv<false>(acc, Ab, Bx, bu, bi, nr);
        __syncthreads();
      }
      trace_mark(a, tk, 1, now_ns());
      for (int idx = threadIdx.x; idx < bu * nr; idx += kThreads) {
        int c = idx / bu, r = idx - c * bu;
        atomicAdd(a.X + rl[r0 + r] + c * a.ldx, -acc[r + c * kT]);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        int last = -1;
        for (int r = 0; r < bu; ++r) {
          int tgt = a.supmember[rl[r0 + r]];
          if (tgt != last) atomicAdd(a.arrived + tgt, 1);
          last = tgt;
        }
      }
      __syncthreads();
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
    if (task.kind == 4) {
      // G: a one-block supernode whole: X_0 -= L_u0^T X_u for every off-diagonal tile
      // (ancestor rows, final once the parent is done), then X_0 <- L_00^-T X_0
      const int w = m.w, noff = (m.h - m.w + kT - 1) / kT;
      const int par = a.sparent[s];
      if (par >= 0 && !wait_geq(a.blkdone + par, (a.meta[par].w + kT - 1) / kT, a.status, s, &sh_ok, a.spin_limit))
        return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(acc, a.X, a.ldx, m.fc, nullptr, w, nr);
      for (int u = 0; u < noff; ++u) {
        const int r0 = w + u * kT, bu = min(kT, m.h - r0);
        __syncthreads();
        stage_block(Ab, P, ld, r0, bu, 0, w);
        stage_x(Bx, a.X, a.ldx, 0, rl + r0, bu, nr);
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
        int c = idx / w, r = idx - c * w;
        a.X[m.fc + r + c * a.ldx] = acc[r + c * kT];
      }
      __syncthreads();
      if (threadIdx.x == 0) red_release(a.blkdone + s, 1);
    } else if (task.kind == 3) {
      // W(u): ancestor rows of tile u, final once the parent is done: X_t -= L_ut^T X_u for
      // every column block t, newest first (the order the diagonal chain needs them)
      const int u = task.t, rr = m.w + u * kT, br = min(kT, m.h - rr);
      const int par = a.sparent[s];
      stage_block(Ab, P, ld, rr, br, (nblk - 1) * kT, m.w - (nblk - 1) * kT);
      if (par >= 0 && !wait_geq(a.blkdone + par, (a.meta[par].w + kT - 1) / kT, a.status, s, &sh_ok, a.spin_limit))
        return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(Bx, a.X, a.ldx, 0, rl + rr, br, nr);
      for (int t = nblk - 1; t >= 0; --t) {
        const int c0 = t * kT, bt = min(kT, m.w - c0);
        if (t < nblk - 1) stage_block(Ab, P, ld, rr, br, c0, bt);
        __syncthreads();
        block_gemv_atomic<true>(a.X, a.ldx, m.fc + c0, Ab, kPld, Bx, bt, br, nr, -1.0);
        __syncthreads();
        if (threadIdx.x == 0) red_release(a.upd + m.boff + t, 1);
      }
    } else if (task.kind == 0) {
      // B(t): every update into X_t has landed; X_t <- L_tt^-T X_t, then X_{t-1} -= L_{t,t-1}^T X_t
      const int t = task.t, c0 = t * kT, bt = min(kT, m.w - c0);
      const int noff = (m.h - m.w + kT - 1) / kT;
      stage_block(Ab, P, ld, c0, bt, c0, bt);  // L is final: load before waiting
      if (t > 0) stage_block<T, kT>(Bx, P, ld, c0, bt, c0 - kT, kT);
      __syncthreads();
      if (threadIdx.x < bt) sh_rinv[threadIdx.x] = 1.0 / Ab[threadIdx.x * (kPld + 1)];
      if (bt == kT) {  // full block: 8 x 8 diagonal inverses, off the chain
        __syncthreads();
        invert_diag8(Ab, sh_rinv);
      }
      if (!wait_geq(a.upd + m.boff + t, noff + nblk - 1 - t, a.status, s, &sh_ok, a.spin_limit)) return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(acc, a.X, a.ldx, m.fc + c0, nullptr, bt, nr);
      __syncthreads();
      if (bt == kT) block_trsv64<false>(acc, Ab, sh_rinv, nr);
      else block_trsv<false>(acc, Ab, sh_rinv, bt, nr);
      __syncthreads();
      for (int idx = threadIdx.x; idx < bt * nr; idx += kThreads) {
        int c = idx / bt, r = idx - c * bt;
        a.X[m.fc + c0 + r + c * a.ldx] = acc[r + c * kT];
      }
      // X_{t-1} -= L_{t,t-1}^T X_t: Bx holds rows c0.. (bt) x columns c0-64.. (64), ld kT
      if (t > 0) block_gemv_atomic<true>(a.X, a.ldx, m.fc + c0 - kT, Bx, kT, acc, kT, bt, nr, -1.0);
      __syncthreads();
      if (threadIdx.x == 0) {
        if (t > 0) red_release(a.upd + m.boff + t - 1, 1);  // the previous block first: it is on the chain
        red_release(a.blkdone + s, 1);
      }
    } else {
      // V(t, u): X_u -= L_tu^T X_t
      const int t = task.i, u = task.t, rr = t * kT, br = min(kT, m.w - rr), c0 = u * kT, bu = min(kT, m.w - c0);
      stage_block(Ab, P, ld, rr, br, c0, bu);
      if (!wait_geq(a.blkdone + s, nblk - t, a.status, s, &sh_ok, a.spin_limit)) return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(Bx, a.X, a.ldx, m.fc + rr, nullptr, br, nr);
      __syncthreads();
      block_gemv_atomic<true>(a.X, a.ldx, m.fc + c0, Ab, kPld, Bx, bu, br, nr, -1.0);
      signal(a.upd + m.boff + u);
    }
    trace_mark(a, tk, 2, now_ns());
  }
}

// ---- dense root solve: one thread-block cluster ----------------------------------
// The root supernode of a nested-dissection tree is a dense w x w lower triangle (the
// 27-point 80^3 stencil's is 21,146 wide), and a sweep over it is a chain of w/64
// diagonal-block solves.  Through global counters each link costs several us; inside
// one cluster it is a barrier.cluster round and a distributed-shared-memory read.
// Block b (64 columns) belongs to cluster rank b % C.  Step t of the forward sweep:
// every CTA copies x_t from its owner's shared memory; the owner of block t+1 first
// subtracts L_{t+1,t} x_t from its rows, solves its diagonal block and publishes
// x_{t+1}; then every CTA subtracts L_it x_t from the other blocks it owns.  The
// backward sweep mirrors it with L^T.  X rows of a block are only ever touched by its
// owner (no atomics); L blocks stream through a cp.async ring ahead of use (L is final,
// so the loads never wait for the chain).  Few right-hand sides only: the updates are
// FP64 FMA work on C SMs.
constexpr int kDenseRhs = 4;       // right-hand sides per launch (the persistent path takes more)
constexpr int kDenseStages = 4;    // L blocks in flight per CTA
constexpr size_t kDenseSmemMax = 227 * 1024;  // dynamic shared memory one CTA may use

__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory"); }
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cluster_size() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
// Generic address of the same shared-memory location in cluster CTA `rank`.
__device__ __forceinline__ const double* map_rank(const double* p, unsigned rank) {
  unsigned long long r;
  asm volatile("mapa.u64 %0, %1, %2;" : "=l"(r) : "l"(p), "r"(rank));
  return reinterpret_cast<const double*>(r);
}
__device__ __forceinline__ void cp_async16_zfill(void* smem, const void* gmem, bool ok) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(ok ? 16 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// 64 x 64 block of T in shared memory, column-major in 16-byte chunks of kC rows; chunk q
// of column k sits at chunk position q ^ (k & 7), so that a warp reading one row across
// 32 columns, or 16 bytes of 8 columns, hits distinct banks.
template <class T>
struct SwzBlock {
  static constexpr int kC = 16 / (int)sizeof(T);
  __device__ static __forceinline__ int at(int r, int k) { return k * kT + (((r / kC) ^ (k & 7)) * kC) + r % kC; }
};

// Dense-sweep item order of one cluster rank: forward, steps t = 0 .. nblk-2 and the
// owned blocks i > t ascending; backward, steps t = nblk-1 .. 1 and the owned blocks
// j < t descending.  (blk = -1 once exhausted.)
template <bool kFwd>
struct DenseItems {
  int nblk, C, rho, t, blk;
  __device__ void first_of_step() {
    for (;;) {
      if (kFwd ? t > nblk - 2 : t < 1) {
        blk = -1;
        return;
      }
      blk = kFwd ? t + 1 + ((rho - (t + 1)) % C + C) % C : t - 1 - (((t - 1) - rho) % C + C) % C;
      if (kFwd ? blk < nblk : blk >= 0) return;
      t += kFwd ? 1 : -1;
    }
  }
  __device__ void start(int n, int c, int r) {
    nblk = n;
    C = c;
    rho = r;
    t = kFwd ? 0 : n - 1;
    first_of_step();
  }
  __device__ void next() {
    blk += kFwd ? C : -C;
    if (kFwd ? blk >= nblk : blk < 0) {
      t += kFwd ? 1 : -1;
      first_of_step();
    }
  }
};

// Shared-memory layout of k_solve_dense (bytes), for `nown` owned blocks of nr right-hand sides.
template <class T>
struct DenseSmem {
  size_t ring, ad, xs, xpub, red, rinv, acc, total;
  __host__ __device__ DenseSmem(int nown, int nr) {
    ring = 0;
    ad = ring + (size_t)kDenseStages * kT * kT * sizeof(T);
    xs = ad + (size_t)kT * kPld * sizeof(double);
    xpub = xs + (size_t)kT * kDenseRhs * sizeof(double);
    red = xpub + (size_t)kT * kDenseRhs * sizeof(double);
    rinv = red + (size_t)4 * kT * kDenseRhs * sizeof(double);
    acc = rinv + (size_t)kT * sizeof(double);
    total = acc + (size_t)nown * kT * nr * sizeof(double);
  }
};

template <class T, bool kFwd>
__global__ void __launch_bounds__(kThreads, 1) k_solve_dense(PSolveArgs a, int s) {
  extern __shared__ __align__(16) unsigned char dsm[];
  const SnMeta m = a.meta[s];
  const T* P = static_cast<const T*>(a.L) + m.off;
  const int64_t ld = m.ld;
  const int nblk = (m.w + kT - 1) / kT, nr = a.nrhs;
  const int C = (int)cluster_size(), rho = (int)cluster_rank(), tid = threadIdx.x;
  const int nown = (nblk + C - 1) / C;
  const DenseSmem<T> lay(nown, nr);
  T* ring = reinterpret_cast<T*>(dsm + lay.ring);
  double* Ad = reinterpret_cast<double*>(dsm + lay.ad);
  double* xs = reinterpret_cast<double*>(dsm + lay.xs);      // x_t of the current step (ld kT)
  double* xpub = reinterpret_cast<double*>(dsm + lay.xpub);  // x of this CTA's last solved block (ld kT)
  double* red = reinterpret_cast<double*>(dsm + lay.red);    // 4 x 64 x kDenseRhs partial sums
  double* rinv = reinterpret_cast<double*>(dsm + lay.rinv);
  double* accown = reinterpret_cast<double*>(dsm + lay.acc);  // X of the owned blocks, nr x 64 each
  double* X = a.X + m.fc;
  const int64_t ldx = a.ldx;
  auto bw = [&](int b) { return min(kT, m.w - b * kT); };
  auto acc_of = [&](int b) { return accown + (size_t)(b / C) * kT * nr; };  // b owned: b % C == rho

  // the owned blocks' rows of X, held here until solved
  for (int lb = 0; lb < nown; ++lb) {
    const int b = rho + lb * C;
    if (b >= nblk) break;
    const int n = bw(b);
    double* acc = accown + (size_t)lb * kT * nr;
    for (int idx = tid; idx < kT * nr; idx += kThreads) {
      const int c = idx / kT, r = idx - c * kT;
      acc[idx] = r < n ? X[b * kT + r + c * ldx] : 0.0;
    }
  }

  // L block of item (t, b): forward L_{b,t} (rows of b, columns of t), backward L_{t,b}
  auto issue = [&](const DenseItems<kFwd>& it, int slot) {
    T* dst = ring + (size_t)slot * kT * kT;
    constexpr int kC = SwzBlock<T>::kC, kChunks = kT * kT / kC;
    const int rb = kFwd ? it.blk : it.t, cb = kFwd ? it.t : it.blk;
    const int nrow = bw(rb), ncol = bw(cb);
    for (int e = tid; e < kChunks; e += kThreads) {
      const int k = e / (kT / kC), q = e - k * (kT / kC), r = q * kC;
      const bool ok = k < ncol && r < nrow;
      const T* src = ok ? P + (int64_t)rb * kT + r + (int64_t)(cb * kT + k) * ld : P;
      cp_async16_zfill(dst + SwzBlock<T>::at(r, k), src, ok);
    }
  };
  // stage diagonal block b (FP64, ld kPld) and its reciprocal diagonal
  auto stage_diag = [&](int b) {
    if (b < 0 || b >= nblk) return;
    stage_block(Ad, P, ld, b * kT, bw(b), b * kT, bw(b));
    __syncthreads();
    if (tid < bw(b)) rinv[tid] = 1.0 / Ad[tid * (kPld + 1)];
    __syncthreads();
  };
  // solve owned diagonal block b in place in its accumulator, publish it and store it in X
  auto solve_diag = [&](int b) {
    const int n = bw(b);
    double* acc = acc_of(b);
    __syncthreads();
    block_trsv<kFwd>(acc, Ad, rinv, n, nr);
    __syncthreads();
    for (int idx = tid; idx < kT * nr; idx += kThreads) {
      const int c = idx / kT, r = idx - c * kT;
      xpub[idx] = r < n ? acc[idx] : 0.0;
      if (r < n) X[b * kT + r + c * ldx] = acc[idx];
    }
  };

  DenseItems<kFwd> prod, cons;
  prod.start(nblk, C, rho);
  cons.start(nblk, C, rho);
#pragma unroll 1
  for (int q = 0; q < kDenseStages - 1; ++q) {
    if (prod.blk >= 0) {
      issue(prod, q);
      prod.next();
    }
    cp_async_commit();
  }
  int nq = 0;  // items consumed
  // consume one item: X_blk -= L x_t (forward) or L^T x_t (backward), in the owned
  // accumulator; xs holds x_t
  auto consume = [&]() {
    cp_async_wait<kDenseStages - 2>();
    __syncthreads();
    if (prod.blk >= 0) {
      issue(prod, (nq + kDenseStages - 1) % kDenseStages);
      prod.next();
    }
    cp_async_commit();
    const T* Lb = ring + (size_t)(nq % kDenseStages) * kT * kT;
    const int lane_i = tid & 63, part = tid >> 6;
    double part_sum[kDenseRhs];
#pragma unroll
    for (int c = 0; c < kDenseRhs; ++c) part_sum[c] = 0.0;
    if (kFwd) {  // row lane_i, columns part*16 ..
#pragma unroll 4
      for (int kk = 0; kk < 16; ++kk) {
        const int k = part * 16 + kk;
        const double l = (double)Lb[SwzBlock<T>::at(lane_i, k)];
#pragma unroll
        for (int c = 0; c < kDenseRhs; ++c)
          if (c < nr) part_sum[c] = fma(l, xs[k + c * kT], part_sum[c]);
      }
    } else {  // column lane_i, rows part*16 ..
#pragma unroll 4
      for (int rr = 0; rr < 16; ++rr) {
        const int r = part * 16 + rr;
        const double l = (double)Lb[SwzBlock<T>::at(r, lane_i)];
#pragma unroll
        for (int c = 0; c < kDenseRhs; ++c)
          if (c < nr) part_sum[c] = fma(l, xs[r + c * kT], part_sum[c]);
      }
    }
#pragma unroll
    for (int c = 0; c < kDenseRhs; ++c) red[(part * kT + lane_i) * kDenseRhs + c] = part_sum[c];
    __syncthreads();
    if (tid < kT * nr) {
      const int c = tid / kT, r = tid - c * kT;
      acc_of(cons.blk)[r + c * kT] -= red[r * kDenseRhs + c] + red[(kT + r) * kDenseRhs + c] +
                                      red[(2 * kT + r) * kDenseRhs + c] + red[(3 * kT + r) * kDenseRhs + c];
    }
    ++nq;
    cons.next();
  };

  // first block solved without any update: forward block 0, backward block nblk-1
  const int b0 = kFwd ? 0 : nblk - 1;
  int mydiag = kFwd ? rho : nblk - 1 - (((nblk - 1) - rho) % C + C) % C;  // next owned diagonal block
  stage_diag(mydiag);
  const bool own_first = b0 % C == rho;
  if (own_first) {
    solve_diag(b0);
    mydiag += kFwd ? C : -C;
  }
  cluster_arrive();
  if (own_first) stage_diag(mydiag);
#pragma unroll 1
  for (int step = 0; step + 1 < nblk; ++step) {
    const int t = kFwd ? step : nblk - 1 - step, tn = kFwd ? t + 1 : t - 1;
    cluster_wait();  // x_t is published
    {
      const double* src = map_rank(xpub, (unsigned)(t % C));
      for (int idx = tid; idx < kT * nr; idx += kThreads) xs[idx] = src[idx];  // rows past the block are 0
    }
    __syncthreads();
    const bool own_next = tn % C == rho;
    if (own_next) {
      consume();  // item (t, tn) is this rank's first item of the step
      solve_diag(tn);
      mydiag += kFwd ? C : -C;
    }
    cluster_arrive();  // own_next: x_tn published; all: done reading x_t
    while (cons.blk >= 0 && cons.t == t) consume();
    if (own_next) stage_diag(mydiag);  // next owned diagonal block, off the chain
  }
  cluster_wait();
  cp_async_wait<0>();
  if (!kFwd && rho == 0 && tid == 0) a.blkdone[s] = nblk;  // the root is done for the persistent sweep
}

int g_solve_grid = 0;
int g_dense_cluster = 0;  // CTAs per dense-root cluster (0 = unavailable)


}  // namespace

int g_solve_grid16 = 0;  // CTAs of the persistent sweeps for <= 16 right-hand sides

void init_solve_attributes() {
  for (auto f : {k_solve_forward<double, 64>, k_solve_backward<double, 64>, k_solve_forward<float, 64>,
                 k_solve_backward<float, 64>})
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem<64>());
  for (auto f : {k_solve_forward<double, 16>, k_solve_backward<double, 16>, k_solve_forward<float, 16>,
                 k_solve_backward<float, 16>})
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem<16>());
  int dev = 0, sms = 0, per = 0, per16 = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_solve_forward<double, 64>, kThreads, solve_smem<64>());
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per16, k_solve_forward<double, 16>, kThreads, solve_smem<16>());
  g_solve_grid = sms * (per > 0 ? per : 1);
  if (g_solve_grid <= 0) g_solve_grid = 148;
  g_solve_grid16 = sms * (per16 > 0 ? per16 : 1);
  if (g_solve_grid16 <= 0) g_solve_grid16 = g_solve_grid;
  // dense-root cluster: 16 CTAs where the GPU can co-schedule them, else 8, else none
  auto set_dense = [](auto f, size_t smem) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  };
  set_dense(k_solve_dense<double, true>, kDenseSmemMax);
  set_dense(k_solve_dense<double, false>, kDenseSmemMax);
  set_dense(k_solve_dense<float, true>, kDenseSmemMax);
  set_dense(k_solve_dense<float, false>, kDenseSmemMax);
  g_dense_cluster = 0;
  for (int c : {16, 8}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = kDenseSmemMax;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_solve_dense<double, true>, &cfg) == cudaSuccess &&
        nclusters > 0) {
      g_dense_cluster = c;
      break;
    }
  }
  cudaGetLastError();  // a refused cluster size is not an error of the handle
}

bool dense_solve_available(int nrhs, int w) {
  if (g_dense_cluster <= 0 || nrhs < 1 || nrhs > kDenseRhs || w <= 0) return false;
  const int nown = ((w + kT - 1) / kT + g_dense_cluster - 1) / g_dense_cluster;
  return DenseSmem<double>(nown, nrhs).total <= kDenseSmemMax;
}

void launch_solve_dense(cudaStream_t st, const PSolveArgs& a, int s, int w, bool forward) {
  const int nown = ((w + kT - 1) / kT + g_dense_cluster - 1) / g_dense_cluster;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(g_dense_cluster);
  cfg.blockDim = dim3(kThreads);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = g_dense_cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (a.fp32) {
    cfg.dynamicSmemBytes = DenseSmem<float>(nown, a.nrhs).total;
    if (forward) cudaLaunchKernelEx(&cfg, k_solve_dense<float, true>, a, s);
    else cudaLaunchKernelEx(&cfg, k_solve_dense<float, false>, a, s);
  } else {
    cfg.dynamicSmemBytes = DenseSmem<double>(nown, a.nrhs).total;
    if (forward) cudaLaunchKernelEx(&cfg, k_solve_dense<double, true>, a, s);
    else cudaLaunchKernelEx(&cfg, k_solve_dense<double, false>, a, s);
  }
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
