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
constexpr size_t kSmemBytes = (size_t)(kT * kPld + 2 * kT * kT) * sizeof(double);

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
// atomics (i < m, c < nr, k < kk); A column-major with leading dimension lda.
template <bool kTrans>
__device__ __forceinline__ void block_gemv_atomic(double* X, int64_t ldx, int x0, const double* A, int lda,
                                                  const double* B, int m, int kk, int nr, double sign) {
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
    if (idx < m * nr && part == 0) atomicAdd(X + x0 + i + c * ldx, sign * s);
    return;
  }
  for (int idx = threadIdx.x; idx < m * nr; idx += kThreads) {
    int c = idx / m, i = idx - c * m;
    double s = 0.0;
    if (kTrans)
      for (int k = 0; k < kk; ++k) s = fma(A[k + i * lda], B[k + c * kT], s);
    else
      for (int k = 0; k < kk; ++k) s = fma(A[i + k * lda], B[k + c * kT], s);
    atomicAdd(X + x0 + i + c * ldx, sign * s);
  }
}

// Lower-triangular solves of a kk x kk block held in A (ld kPld) against the
// right-hand sides acc (ld kT), one warp per right-hand side column; rinv holds
// the reciprocals of the diagonal (computed off the dependency chain).
// forward: acc <- D^-1 acc ; backward: acc <- D^-T acc.
template <bool kForward>
__device__ void block_trsv(double* acc, const double* A, const double* rinv, int kk, int nr) {
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
        if (lane > k && lane < kk) v0 = fma(-A[lane + k * kPld], xk, v0);
        if (lane + 32 > k && lane + 32 < kk) v1 = fma(-A[lane + 32 + k * kPld], xk, v1);
      } else {
        // rows j < k: acc_j -= D[k][j] x_k
        if (lane < k) v0 = fma(-A[k + lane * kPld], xk, v0);
        if (lane + 32 < k) v1 = fma(-A[k + (lane + 32) * kPld], xk, v1);
      }
    }
    if (lane < kk) acc[lane + c * kT] = v0;
    if (lane + 32 < kk) acc[lane + 32 + c * kT] = v1;
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

template <class T>
__global__ void __launch_bounds__(kThreads) k_solve_forward(PSolveArgs a) {
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
      if (!wait_geq(a.arrived + s, a.expected[s], a.status, s, &sh_ok, a.spin_limit)) return;
      if (!wait_geq(a.upd + m.boff + t, t, a.status, s, &sh_ok, a.spin_limit)) return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(acc, a.X, a.ldx, m.fc + r0, nullptr, bt, nr);
      __syncthreads();
      block_trsv<true>(acc, Ab, sh_rinv, bt, nr);
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
    } else {
      // O(u): off-diagonal rows, Y_K[rows] -= L_KJ Y_J accumulated over the column blocks
      const int u = task.t, r0 = m.w + u * kT, bu = min(kT, m.h - r0);
      const int nblk = (m.w + kT - 1) / kT;
      for (int idx = threadIdx.x; idx < kT * nr; idx += kThreads) acc[idx] = 0.0;
      for (int i = 0; i < nblk; ++i) {
        const int bi = min(kT, m.w - i * kT);
        stage_block(Ab, P, ld, r0, bu, i * kT, bi);
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

template <class T>
__global__ void __launch_bounds__(kThreads) k_solve_backward(PSolveArgs a) {
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
    if (task.kind == 3) {
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
      if (!wait_geq(a.upd + m.boff + t, noff + nblk - 1 - t, a.status, s, &sh_ok, a.spin_limit)) return;
      trace_mark(a, tk, 1, now_ns());
      stage_x(acc, a.X, a.ldx, m.fc + c0, nullptr, bt, nr);
      __syncthreads();
      block_trsv<false>(acc, Ab, sh_rinv, bt, nr);
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

int g_solve_grid = 0;

}  // namespace

void init_solve_attributes() {
  for (auto f : {k_solve_forward<double>, k_solve_backward<double>, k_solve_forward<float>, k_solve_backward<float>})
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_solve_forward<double>, kThreads, kSmemBytes);
  g_solve_grid = sms * (per > 0 ? per : 1);
  if (g_solve_grid <= 0) g_solve_grid = 148;
}

void launch_solve_persistent(cudaStream_t st, const PSolveArgs& a, bool forward) {
  if (a.ntasks <= 0 || a.spin_limit <= 0) return;
  int grid = g_solve_grid < a.ntasks ? g_solve_grid : a.ntasks;
  if (a.fp32) {
    if (forward) k_solve_forward<float><<<grid, kThreads, kSmemBytes, st>>>(a);
    else k_solve_backward<float><<<grid, kThreads, kSmemBytes, st>>>(a);
  } else {
    if (forward) k_solve_forward<double><<<grid, kThreads, kSmemBytes, st>>>(a);
    else k_solve_backward<double><<<grid, kThreads, kSmemBytes, st>>>(a);
  }
}

}  // namespace dev
}  // namespace spb
