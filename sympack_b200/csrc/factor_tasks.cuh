// Device bodies of the panel tasks of the supernodal factorization (sm_100a),
// shared by the per-step kernels (kernels.cu) and the persistent factorization
// kernel (gemm.cu).  Every body works with the whole thread block (any multiple of
// 32 threads for the small panel, 256 for the others) and the shared memory it is given.
//
// Numerics follow symPACK's blockCell_t operations (symPACKMatrix2D.hpp):
//   factorize   1052-1102  Potrf of the diagonal block
//   trsm        1104-1178  L_KI = A_KI * L_II^-T
// on a column-major panel per supernode instead of row-major cells.
// LDL^T (blockCellLDL_t, 2D.hpp:1802-2465): Potrf_LDL of the diagonal block
// (lapack.hpp:206-560, no pivoting, a zero pivot is reported), unit TRSM then
// scaling by 1/D (2D.hpp:2118-2137).
#pragma once
#include <type_traits>
#include "kernels.cuh"

namespace spb {
namespace dev {
namespace ftask {
namespace {

__device__ __forceinline__ void report(Status* st, int code, int s, int col) {
  if (atomicCAS(&st->code, 0, code) == 0) {
    st->supernode = s;
    st->column = col;
  }
}

// Unblocked right-looking Cholesky of an h x w column-major panel held in
// shared memory (leading dimension ldp): the w x w top block becomes L_II and
// the rows below become L_KI = A_KI L_II^-T.  All threads of the block take part.
__device__ void panel_cholesky_smem(double* P, int h, int w, int ldp, Status* status, int s, int fc) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int warp = tid >> 5, lane = tid & 31, nw = nthr >> 5;
  for (int k = 0; k < w; ++k) {
    if (tid == 0) {
      double d = P[k + k * ldp];
      if (!(d > 0.0)) {
        if (status) report(status, 1, s, fc + k);
        d = 1.0;
      }
      P[k + k * ldp] = sqrt(d);
    }
    __syncthreads();
    const double inv = 1.0 / P[k + k * ldp];
    for (int i = k + 1 + tid; i < h; i += nthr) P[i + k * ldp] *= inv;
    __syncthreads();
    for (int j = k + 1 + warp; j < w; j += nw) {
      const double ljk = P[j + k * ldp];
      for (int i = j + lane; i < h; i += 32) P[i + j * ldp] -= P[i + k * ldp] * ljk;
    }
    __syncthreads();
  }
}

// LDL^T counterpart: the w x w top block becomes unit L_II with D on its diagonal,
// the rows below L_KI = A_KI L_II^-T D^-1.  Column k's trailing update uses the
// column before it is scaled (A_ij -= A_ik A_jk / d_k).  A zero pivot is reported
// (status 1) and replaced by 1 so that the factorization runs to its end.
__device__ void panel_ldl_smem(double* P, int h, int w, int ldp, Status* status, int s, int fc) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int warp = tid >> 5, lane = tid & 31, nw = nthr >> 5;
  for (int k = 0; k < w; ++k) {
    if (tid == 0) {
      const double d = P[k + k * ldp];
      if (!(fabs(d) > 0.0)) {
        if (status) report(status, 1, s, fc + k);
        P[k + k * ldp] = 1.0;
      }
    }
    __syncthreads();
    const double dinv = 1.0 / P[k + k * ldp];
    for (int j = k + 1 + warp; j < w; j += nw) {
      const double ljk = P[j + k * ldp] * dinv;
      for (int i = j + lane; i < h; i += 32) P[i + j * ldp] -= P[i + k * ldp] * ljk;
    }
    __syncthreads();
    for (int i = k + 1 + tid; i < h; i += nthr) P[i + k * ldp] *= dinv;
    __syncthreads();
  }
}

// Split copy of final FP32 panel rows (TMA-fed tcgen05 tiles): tf32 hi part (round to
// nearest, ties away) and the rounded remainder, row-major, hi block then lo block.
__device__ __forceinline__ void split_store(const FactorArgs& a, const SnMeta& m, int64_t off, int r, int c, float x) {
  uint32_t hi, lo;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(x - __uint_as_float(hi)));
  const int64_t pitch = (m.w + 3) & ~3;
  float* p = a.split + off + (int64_t)r * pitch + c;
  p[0] = __uint_as_float(hi);
  p[(int64_t)m.h * pitch] = __uint_as_float(lo);
}
// The copy's writes come before the TMA loads (async proxy) of the tasks that wait for
// this one's counters.
__device__ __forceinline__ void split_fence() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// Small panel s factored whole in shared memory P (h * w doubles).
template <class T>
__device__ __noinline__ void factor_small_task(const FactorArgs& a, int s, double* P) {
  const SnMeta m = a.meta[s];
  const int h = m.h, w = m.w;
  T* g = static_cast<T*>(a.L) + m.off;
  for (int idx = threadIdx.x; idx < h * w; idx += blockDim.x) {
    int c = idx / h, r = idx - c * h;
    P[idx] = (double)g[r + (int64_t)c * m.ld];
  }
  __syncthreads();
  if (a.ldl) {
    panel_ldl_smem(P, h, w, h, a.status, s, m.fc);
    double* gw = a.W + m.off;
    for (int idx = threadIdx.x; idx < h * w; idx += blockDim.x) {
      const int c = idx / h, r = idx - c * h;
      const double v = P[idx], d = P[c + c * h];
      g[r + (int64_t)c * m.ld] = (T)(r == c ? 1.0 : v);
      gw[r + (int64_t)c * m.ld] = r == c ? d : (r > c ? v * d : 0.0);
    }
    return;
  }
  panel_cholesky_smem(P, h, w, h, a.status, s, m.fc);
  for (int idx = threadIdx.x; idx < h * w; idx += blockDim.x) {
    int c = idx / h, r = idx - c * h;
    g[r + (int64_t)c * m.ld] = (T)P[idx];
  }
  if constexpr (std::is_same<T, float>::value) {
    const int64_t off = a.split ? a.split_off[s] : -1;
    if (off >= 0) {  // off-diagonal rows, row by row (consecutive threads take consecutive columns)
      for (int idx = threadIdx.x; idx < (h - w) * w; idx += blockDim.x) {
        const int r = w + idx / w, c = idx % w;
        split_store(a, m, off, r, c, (float)P[r + c * h]);
      }
      split_fence();
    }
  }
}

constexpr int kNB = 64;
constexpr int kThreads = 256;  // threads of the POTRF and TRSM kernels

// POTRF of one 64-column diagonal block [c0, c0+nb) of a wide panel (one CTA
// per item), right-looking by 8-column pieces in shared memory.  Every thread factors
// the 8 x 8 diagonal piece itself, in registers, from the same shared-memory values (the
// same operations in the same order, so every copy is identical): no shuffles and no
// barrier between the piece and the solve of the rows below, which each thread then
// does for its own row against its register copy.  The factored pieces go to a side
// array (other threads may still be reading the unfactored piece) and into the block at
// the end.  The trailing lower triangle is updated with the solved columns (thread
// (row, group) updates columns group, group+4, ... of its row).  Two barriers per
// piece.  The CTA also copies the factored block (FP64) and 1/L_kk to its scratch
// slot, from where the TRSM of the rows below reads them.  A block narrower than 64 is
// padded with the identity.  The kernel sits on the critical path of every wide
// supernode and is latency-bound.
constexpr int kDL = kNB + 1;  // padded leading dimension in shared memory
// scratch slot: factored block (FP64), 1/L_kk, and (LDL^T) 1/D_kk
constexpr size_t kSlot = kDiagSlotDoubles;
static_assert(kSlot >= (size_t)kNB * kNB + 2 * kNB, "slot layout");
constexpr int kPiece = 8;
constexpr int kTri = kPiece * (kPiece + 1) / 2;  // entries of a lower-triangular piece
__host__ __device__ constexpr int tri(int i, int j) { return i * (i + 1) / 2 + j; }  // i >= j

// Shared memory (doubles) of potrf_diag_task and ldl_diag_task.
constexpr int kDiagSmemDoubles = kNB * kDL + (kNB / kPiece) * kTri + kNB * kPiece + kNB;

template <class T>
__device__ __noinline__ void potrf_diag_task(const FactorArgs& a, const PanelItem& it, double* __restrict__ winv, double* sm) {
  double* D = sm;
  double(*Lp)[kTri] = reinterpret_cast<double(*)[kTri]>(sm + kNB * kDL);  // factored diagonal pieces
  double* Rinv = sm + kNB * kDL + (kNB / kPiece) * kTri;                  // 1 / L_kk
  const SnMeta m = a.meta[it.s];
  const T* g = static_cast<const T*>(a.L) + m.off;
  const int nb = it.nb, c0 = it.c0;
  const int64_t ld = m.ld;
  const int tid = threadIdx.x;
  {
    double v[kNB * kNB / kThreads];
#pragma unroll
    for (int q = 0; q < kNB * kNB / kThreads; ++q) {
      const int idx = tid + q * kThreads, c = idx / kNB, r = idx - c * kNB;
      v[q] = (r < nb && c < nb && r >= c) ? (double)g[(c0 + r) + (int64_t)(c0 + c) * ld] : (r == c ? 1.0 : 0.0);
    }
#pragma unroll
    for (int q = 0; q < kNB * kNB / kThreads; ++q) {
      const int idx = tid + q * kThreads, c = idx / kNB, r = idx - c * kNB;
      D[r + c * kDL] = v[q];
    }
  }
  __syncthreads();
  const int urow = tid & 63, ugrp = tid >> 6;  // update mapping: row kb+8+urow, columns kb+8+ugrp+4t
#pragma unroll 1
  for (int kb = 0; kb < kNB; kb += kPiece) {
    // the 8 x 8 piece, factored by every thread
    double l[kTri], rs[kPiece];
#pragma unroll
    for (int i = 0; i < kPiece; ++i)
#pragma unroll
      for (int j = 0; j <= i; ++j) l[tri(i, j)] = D[kb + i + (kb + j) * kDL];
#pragma unroll
    for (int k = 0; k < kPiece; ++k) {
      double dkk = l[tri(k, k)];
      if (!(dkk > 0.0)) {
        if (tid == 0 && kb + k < nb) report(a.status, 1, it.s, m.fc + c0 + kb + k);
        dkk = 1.0;
      }
      rs[k] = rsqrt(dkk);
      l[tri(k, k)] = dkk * rs[k];
#pragma unroll
      for (int i = k + 1; i < kPiece; ++i) l[tri(i, k)] *= rs[k];
#pragma unroll
      for (int j = k + 1; j < kPiece; ++j)
#pragma unroll
        for (int i = j; i < kPiece; ++i) l[tri(i, j)] = fma(-l[tri(i, k)], l[tri(j, k)], l[tri(i, j)]);
    }
    if (tid < kTri) {
      double mine = 0.0;
#pragma unroll
      for (int e = 0; e < kTri; ++e)
        if (e == tid) mine = l[e];
      Lp[kb / kPiece][tid] = mine;
    }
    if (tid < kPiece) {
      double mine = 0.0;
#pragma unroll
      for (int e = 0; e < kPiece; ++e)
        if (e == tid) mine = rs[e];
      Rinv[kb + tid] = mine;
    }
    const int below = kNB - kb - kPiece;
    if (below == 0) break;
    if (tid < below) {  // one row per thread: solve against the piece
      const int i = kb + kPiece + tid;
      double x[kPiece];
#pragma unroll
      for (int j = 0; j < kPiece; ++j) x[j] = D[i + (kb + j) * kDL];
#pragma unroll
      for (int k = 0; k < kPiece; ++k) {
        double t = x[k];
#pragma unroll
        for (int j = 0; j < k; ++j) t = fma(-x[j], l[tri(k, j)], t);
        x[k] = t * rs[k];
      }
#pragma unroll
      for (int j = 0; j < kPiece; ++j) D[i + (kb + j) * kDL] = x[j];
    }
    __syncthreads();
    if (urow < below) {
      const int i = kb + kPiece + urow;
      double x[kPiece];
#pragma unroll
      for (int k = 0; k < kPiece; ++k) x[k] = D[i + (kb + k) * kDL];
      for (int j = kb + kPiece + ugrp; j <= i; j += 4) {
        double t0 = D[i + j * kDL], t1 = 0.0;
#pragma unroll
        for (int k = 0; k < kPiece; k += 2) {
          t0 = fma(-x[k], D[j + (kb + k) * kDL], t0);
          t1 = fma(-x[k + 1], D[j + (kb + k + 1) * kDL], t1);
        }
        D[i + j * kDL] = t0 + t1;
      }
    }
    __syncthreads();
  }
  __syncthreads();
  // factored pieces into the block
  for (int e = tid; e < (kNB / kPiece) * kTri; e += kThreads) {
    const int p = e / kTri, q = e - p * kTri;
    int i = 0;
    while (tri(i + 1, 0) <= q) ++i;
    const int j = q - tri(i, 0);
    D[p * kPiece + i + (p * kPiece + j) * kDL] = Lp[p][q];
  }
  __syncthreads();
  T* gw = static_cast<T*>(a.L) + m.off;
#pragma unroll
  for (int q = 0; q < kNB * kNB / kThreads; ++q) {
    const int idx = tid + q * kThreads, c = idx / kNB, r = idx - c * kNB;
    if (r < nb && c < nb && r >= c) gw[(c0 + r) + (int64_t)(c0 + c) * ld] = (T)D[r + c * kDL];
  }
  // FP64 copy of the factored block and 1/L_kk for the TRSM of the rows below
  if (winv) {
    double* W = winv + (size_t)it.slot * kSlot;
#pragma unroll
    for (int q = 0; q < kNB * kNB / kThreads; ++q) {
      const int idx = tid + q * kThreads, c = idx / kNB, r = idx - c * kNB;
      W[idx] = D[r + c * kDL];
    }
    if (tid < kNB) W[kNB * kNB + tid] = Rinv[tid];
  }
}

// LDL^T of one 64-column diagonal block [c0, c0+nb) (one CTA per item), right-looking by
// 8-column pieces like potrf_diag_task: every thread factors the piece itself in registers
// (Potf2_LDL, lapack.hpp:206-270, on the lower triangle: d_k = A_kk, |d_k| > 0 or the
// pivot is reported as a zero pivot; column k is divided by d_k; A_ij loses L_ik A_jk),
// then each row below solves w = r L^-T against the unit piece (w is that row of L D)
// and stores r's L values w / d; the trailing triangle loses W_ik L_jk.  L takes the
// unit block, W the block times D (its diagonal is D), the scratch slot the unit block,
// 1 in place of 1/L_kk (the TRSM of the rows below then computes R L11^-T, which is W's
// rows) and 1/D_kk.
template <class T>
__device__ __noinline__ void ldl_diag_task(const FactorArgs& a, const PanelItem& it, double* __restrict__ winv, double* sm) {
  double* D = sm;
  double(*Lp)[kTri] = reinterpret_cast<double(*)[kTri]>(sm + kNB * kDL);  // unit L below, d on the diagonal
  double* Wr = sm + kNB * kDL + (kNB / kPiece) * kTri;                    // rows below the piece: W = L D, ld kNB
  double* Dk = Wr + kNB * kPiece;
  const SnMeta m = a.meta[it.s];
  T* g = static_cast<T*>(a.L) + m.off;
  const int nb = it.nb, c0 = it.c0;
  const int64_t ld = m.ld;
  const int tid = threadIdx.x;
  {
    double v[kNB * kNB / kThreads];
#pragma unroll
    for (int q = 0; q < kNB * kNB / kThreads; ++q) {
      const int idx = tid + q * kThreads, c = idx / kNB, r = idx - c * kNB;
      v[q] = (r < nb && c < nb && r >= c) ? (double)g[(c0 + r) + (int64_t)(c0 + c) * ld] : (r == c ? 1.0 : 0.0);
    }
#pragma unroll
    for (int q = 0; q < kNB * kNB / kThreads; ++q) {
      const int idx = tid + q * kThreads, c = idx / kNB, r = idx - c * kNB;
      D[r + c * kDL] = v[q];
    }
  }
  __syncthreads();
  const int urow = tid & 63, ugrp = tid >> 6;
#pragma unroll 1
  for (int kb = 0; kb < kNB; kb += kPiece) {
    double l[kTri], dinv[kPiece];
#pragma unroll
    for (int i = 0; i < kPiece; ++i)
#pragma unroll
      for (int j = 0; j <= i; ++j) l[tri(i, j)] = D[kb + i + (kb + j) * kDL];
#pragma unroll
    for (int k = 0; k < kPiece; ++k) {
      double d = l[tri(k, k)];
      if (!(fabs(d) > 0.0)) {
        if (tid == 0 && kb + k < nb) report(a.status, 1, it.s, m.fc + c0 + kb + k);
        d = 1.0;
        l[tri(k, k)] = 1.0;
      }
      dinv[k] = 1.0 / d;
      double w[kPiece];
#pragma unroll
      for (int i = k + 1; i < kPiece; ++i) {
        w[i] = l[tri(i, k)];
        l[tri(i, k)] = w[i] * dinv[k];
      }
#pragma unroll
      for (int j = k + 1; j < kPiece; ++j)
#pragma unroll
        for (int i = j; i < kPiece; ++i) l[tri(i, j)] = fma(-l[tri(i, k)], w[j], l[tri(i, j)]);
    }
    if (tid < kTri) {
      double mine = 0.0;
#pragma unroll
      for (int e = 0; e < kTri; ++e)
        if (e == tid) mine = l[e];
      Lp[kb / kPiece][tid] = mine;
    }
    if (tid < kPiece) {
      double mine = 0.0;
#pragma unroll
      for (int e = 0; e < kPiece; ++e)
        if (e == tid) mine = l[tri(e, e)];
      Dk[kb + tid] = mine;
    }
    const int below = kNB - kb - kPiece;
    if (below == 0) break;
    if (tid < below) {  // one row per thread: w = r L^-T (unit piece), L row = w / d
      const int i = kb + kPiece + tid;
      double x[kPiece];
#pragma unroll
      for (int j = 0; j < kPiece; ++j) x[j] = D[i + (kb + j) * kDL];
#pragma unroll
      for (int k = 0; k < kPiece; ++k) {
        double t = x[k];
#pragma unroll
        for (int j = 0; j < k; ++j) t = fma(-x[j], l[tri(k, j)], t);
        x[k] = t;
      }
#pragma unroll
      for (int j = 0; j < kPiece; ++j) {
        Wr[i + j * kNB] = x[j];
        D[i + (kb + j) * kDL] = x[j] * dinv[j];
      }
    }
    __syncthreads();
    if (urow < below) {
      const int i = kb + kPiece + urow;
      double x[kPiece];
#pragma unroll
      for (int k = 0; k < kPiece; ++k) x[k] = Wr[i + k * kNB];
      for (int j = kb + kPiece + ugrp; j <= i; j += 4) {
        double t0 = D[i + j * kDL], t1 = 0.0;
#pragma unroll
        for (int k = 0; k < kPiece; k += 2) {
          t0 = fma(-x[k], D[j + (kb + k) * kDL], t0);
          t1 = fma(-x[k + 1], D[j + (kb + k + 1) * kDL], t1);
        }
        D[i + j * kDL] = t0 + t1;
      }
    }
    __syncthreads();
  }
  __syncthreads();
  for (int e = tid; e < (kNB / kPiece) * kTri; e += kThreads) {
    const int p = e / kTri, q = e - p * kTri;
    int i = 0;
    while (tri(i + 1, 0) <= q) ++i;
    const int j = q - tri(i, 0);
    D[p * kPiece + i + (p * kPiece + j) * kDL] = i == j ? 1.0 : Lp[p][q];
  }
  __syncthreads();
  double* gw = a.W + m.off;
#pragma unroll
  for (int q = 0; q < kNB * kNB / kThreads; ++q) {
    const int idx = tid + q * kThreads, c = idx / kNB, r = idx - c * kNB;
    if (r < nb && c < nb && r >= c) {
      const double l = D[r + c * kDL];
      g[(c0 + r) + (int64_t)(c0 + c) * ld] = (T)l;
      gw[(c0 + r) + (int64_t)(c0 + c) * ld] = r == c ? Dk[c] : l * Dk[c];
    }
  }
  if (winv) {
    double* S = winv + (size_t)it.slot * kSlot;
#pragma unroll
    for (int q = 0; q < kNB * kNB / kThreads; ++q) {
      const int idx = tid + q * kThreads, c = idx / kNB, r = idx - c * kNB;
      S[idx] = D[r + c * kDL];
    }
    if (tid < kNB) {
      S[kNB * kNB + tid] = 1.0;
      S[kNB * kNB + kNB + tid] = 1.0 / Dk[tid];
    }
  }
}

// TRSM of one 64-row tile below a factored diagonal block, R <- R L11^-T, by
// 8-column pieces: each row solves against the 8 x 8 diagonal piece (one
// thread per row), then the remaining columns of the tile are updated with the
// solved piece (thread (row, group) takes columns group, group+4, ...).  L11
// and 1/L_kk come from the scratch slot.  All loads are issued before the first
// use (32 per thread in flight).
// Shared memory (doubles) of trsm_rows_task.
constexpr int kTrsmSmemDoubles = 2 * kNB * kDL + kNB;

template <class T>
__device__ __noinline__ void trsm_rows_task(const FactorArgs& a, const PanelItem& it, const double* __restrict__ winv,
                               double* sm) {
  double* R = sm;                // R[r + k*kDL]
  double* D = sm + kNB * kDL;    // D[i + j*kDL] = L11[i][j]
  double* Rinv = sm + 2 * kNB * kDL;
  const SnMeta m = a.meta[it.s];
  T* g = static_cast<T*>(a.L) + m.off;
  const int nb = it.nb, c0 = it.c0;
  const int64_t ld = m.ld;
  const int rows = min(kNB, m.h - it.row0);
  const double* W = winv + (size_t)it.slot * kSlot;
  const int tid = threadIdx.x;
  {
    double v[kNB * kNB / kThreads], w[kNB * kNB / kThreads];
#pragma unroll
    for (int q = 0; q < kNB * kNB / kThreads; ++q) {
      const int idx = tid + q * kThreads, k = idx / kNB, r = idx - k * kNB;
      v[q] = (r < rows && k < nb) ? (double)g[(it.row0 + r) + (int64_t)(c0 + k) * ld] : 0.0;
      w[q] = W[idx];
    }
#pragma unroll
    for (int q = 0; q < kNB * kNB / kThreads; ++q) {
      const int idx = tid + q * kThreads, k = idx / kNB, r = idx - k * kNB;
      R[r + k * kDL] = v[q];
      D[r + k * kDL] = w[q];
    }
  }
  if (tid < kNB) Rinv[tid] = W[kNB * kNB + tid];
  __syncthreads();
  const int urow = tid & 63, ugrp = tid >> 6;
#pragma unroll 1
  for (int kb = 0; kb < nb; kb += kPiece) {
    if (tid < rows) {
      double x[kPiece];
#pragma unroll
      for (int j = 0; j < kPiece; ++j) x[j] = R[tid + (kb + j) * kDL];
#pragma unroll
      for (int k = 0; k < kPiece; ++k) {
        double t = x[k];
#pragma unroll
        for (int j = 0; j < k; ++j) t = fma(-x[j], D[kb + k + (kb + j) * kDL], t);
        x[k] = t * Rinv[kb + k];
      }
#pragma unroll
      for (int j = 0; j < kPiece; ++j) R[tid + (kb + j) * kDL] = x[j];
    }
    __syncthreads();
    if (kb + kPiece >= nb) break;
    if (urow < rows) {
      double x[kPiece];
#pragma unroll
      for (int k = 0; k < kPiece; ++k) x[k] = R[urow + (kb + k) * kDL];
      for (int j = kb + kPiece + ugrp; j < nb; j += 4) {
        double t0 = R[urow + j * kDL], t1 = 0.0;
#pragma unroll
        for (int k = 0; k < kPiece; k += 2) {
          t0 = fma(-x[k], D[j + (kb + k) * kDL], t0);
          t1 = fma(-x[k + 1], D[j + (kb + k + 1) * kDL], t1);
        }
        R[urow + j * kDL] = t0 + t1;
      }
    }
    __syncthreads();
  }
  if (a.ldl) {  // R is W's rows (R L11^-T with unit L11); L's rows are R D^-1
    const double* dinv = W + kNB * kNB + kNB;
    double* gw = a.W + m.off;
#pragma unroll
    for (int q = 0; q < kNB * kNB / kThreads; ++q) {
      const int idx = tid + q * kThreads, k = idx / kNB, r = idx - k * kNB;
      if (r < rows && k < nb) {
        const double v = R[r + k * kDL];
        g[(it.row0 + r) + (int64_t)(c0 + k) * ld] = (T)(v * dinv[k]);
        gw[(it.row0 + r) + (int64_t)(c0 + k) * ld] = v;
      }
    }
    return;
  }
#pragma unroll
  for (int q = 0; q < kNB * kNB / kThreads; ++q) {
    const int idx = tid + q * kThreads, k = idx / kNB, r = idx - k * kNB;
    if (r < rows && k < nb) g[(it.row0 + r) + (int64_t)(c0 + k) * ld] = (T)R[r + k * kDL];
  }
  if constexpr (std::is_same<T, float>::value) {
    const int64_t off = a.split ? a.split_off[it.s] : -1;
    if (off >= 0) {  // the tile's rows, row by row (consecutive threads take consecutive columns)
#pragma unroll
      for (int q = 0; q < kNB * kNB / kThreads; ++q) {
        const int idx = tid + q * kThreads, r = idx / kNB, k = idx - r * kNB;
        if (r < rows && k < nb) split_store(a, m, off, it.row0 + r, c0 + k, (float)R[r + k * kDL]);
      }
      split_fence();
    }
  }
}


}  // namespace
}  // namespace ftask
}  // namespace dev
}  // namespace spb
