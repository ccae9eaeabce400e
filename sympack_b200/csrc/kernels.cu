// Supernodal Cholesky factor and solve kernels for sm_100a.
//
// Numerics follow symPACK's blockCell_t operations (symPACKMatrix2D.hpp):
//   factorize   1052-1102  Potrf of the diagonal block
//   trsm        1104-1178  L_KI = A_KI * L_II^-T
//   update      1180-1469  target(K,J) -= L_KI * L_JI^T, scattered through row/column maps
//   forward_update / forward_update_contrib   1486-1643
//   back_update / _tri_solve / back_update_contrib   1645-1797
// on a column-major panel per supernode instead of row-major cells.
#include <cfloat>
#include <climits>
#include <cstdio>

#include "kernels.cuh"

namespace spb {
namespace dev {

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

__global__ void k_assemble(double* __restrict__ L, const int64_t* __restrict__ dst,
                           const double* __restrict__ vals, int64_t nnz) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x)
    L[dst[i]] = vals[i];
}

__global__ void __launch_bounds__(128) k_factor_small(FactorArgs a, const int32_t* __restrict__ items) {
  extern __shared__ double P[];
  const int s = items[blockIdx.x];
  const SnMeta m = a.meta[s];
  const int h = m.h, w = m.w;
  double* g = a.L + m.off;
  for (int idx = threadIdx.x; idx < h * w; idx += blockDim.x) {
    int c = idx / h, r = idx - c * h;
    P[idx] = g[r + (int64_t)c * m.ld];
  }
  __syncthreads();
  panel_cholesky_smem(P, h, w, h, a.status, s, m.fc);
  for (int idx = threadIdx.x; idx < h * w; idx += blockDim.x) {
    int c = idx / h, r = idx - c * h;
    g[r + (int64_t)c * m.ld] = P[idx];
  }
}

constexpr int kNB = 64;

// POTRF of one diagonal block [c0, c0+nb) of a wide panel (one CTA per item).
__global__ void __launch_bounds__(256) k_potrf_diag(FactorArgs a, const PanelItem* __restrict__ items) {
  __shared__ double D[kNB * kNB];
  const PanelItem it = items[blockIdx.x];
  const SnMeta m = a.meta[it.s];
  double* g = a.L + m.off;
  const int nb = it.nb, c0 = it.c0;
  const int64_t ld = m.ld;
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    int c = idx / nb, r = idx - c * nb;
    D[r + c * kNB] = (r >= c) ? g[(c0 + r) + (int64_t)(c0 + c) * ld] : 0.0;
  }
  __syncthreads();
  panel_cholesky_smem(D, nb, nb, kNB, a.status, it.s, m.fc + c0);
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    int c = idx / nb, r = idx - c * nb;
    if (r >= c) g[(c0 + r) + (int64_t)(c0 + c) * ld] = D[r + c * kNB];
  }
}

// TRSM of one 128-row tile below a factored 64-column diagonal block:
// R <- R D^-T.  One thread per row; the row lives in registers and is solved
// by forward substitution against D broadcast from shared memory.
__global__ void __launch_bounds__(128) k_trsm_rows(FactorArgs a, const PanelItem* __restrict__ items) {
  __shared__ double D[kNB * kNB];  // row-major: D[k * kNB + j], zero above the diagonal and past nb
  __shared__ double Dinv[kNB];
  const PanelItem it = items[blockIdx.x];
  const SnMeta m = a.meta[it.s];
  double* g = a.L + m.off;
  const int nb = it.nb, c0 = it.c0;
  const int64_t ld = m.ld;
  for (int idx = threadIdx.x; idx < kNB * kNB; idx += blockDim.x) {
    int k = idx / kNB, j = idx - k * kNB;
    D[idx] = (k < nb && j <= k) ? g[(c0 + k) + (int64_t)(c0 + j) * ld] : 0.0;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < kNB; k += blockDim.x) Dinv[k] = k < nb ? 1.0 / D[k * kNB + k] : 0.0;
  __syncthreads();
  const int r = threadIdx.x;
  if (it.row0 + r >= m.h) return;
  double x[kNB];
  {
    const double* p = g + it.row0 + r + (int64_t)c0 * ld;
#pragma unroll
    for (int j = 0; j < kNB; ++j, p += ld) x[j] = j < nb ? *p : 0.0;
  }
#pragma unroll
  for (int k = 0; k < kNB; ++k) {
    double s0 = x[k], s1 = 0.0;
#pragma unroll
    for (int j = 0; j + 1 < k; j += 2) {
      s0 = fma(-x[j], D[k * kNB + j], s0);
      s1 = fma(-x[j + 1], D[k * kNB + j + 1], s1);
    }
    if (k & 1) s0 = fma(-x[k - 1], D[k * kNB + k - 1], s0);
    x[k] = (s0 + s1) * Dinv[k];
  }
  // a fresh pointer walk for the stores (keeps 64 addresses from living across the solve)
  double* q = g + it.row0 + r;
  asm volatile("" : "+l"(q));
  q += (int64_t)c0 * ld;
#pragma unroll
  for (int j = 0; j < kNB; ++j, q += ld)
    if (j < nb) *q = x[j];
}

__global__ void k_permute_in(double* X, int64_t ldx, const double* B, int64_t ldb, const int32_t* invp0, int n,
                             int nrhs) {
  int64_t total = (int64_t)n * nrhs;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int c = (int)(i / n), r = (int)(i - (int64_t)c * n);
    X[invp0[r] + c * ldx] = B[r + c * ldb];
  }
}

__global__ void k_permute_out(double* B, int64_t ldb, const double* X, int64_t ldx, const int32_t* invp0, int n,
                              int nrhs) {
  int64_t total = (int64_t)n * nrhs;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int c = (int)(i / n), r = (int)(i - (int64_t)c * n);
    B[r + c * ldb] = X[invp0[r] + c * ldx];
  }
}

int grid_for(int64_t work, int threads) {
  int64_t g = (work + threads - 1) / threads;
  if (g > 148 * 16) g = 148 * 16;
  return g < 1 ? 1 : (int)g;
}

}  // namespace

void launch_assemble(cudaStream_t st, double* L, const int64_t* dst, const double* vals, int64_t nnz) {
  if (nnz <= 0) return;
  k_assemble<<<grid_for(nnz, 256), 256, 0, st>>>(L, dst, vals, nnz);
}

void init_kernel_attributes() {
  init_gemm_attributes();
  init_solve_attributes();
  cudaFuncSetAttribute(k_factor_small, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
}

void launch_factor_small(cudaStream_t st, const FactorArgs& a, const int32_t* items, int count, int smem_bytes) {
  k_factor_small<<<count, 128, smem_bytes, st>>>(a, items);
}

void launch_potrf_diag(cudaStream_t st, const FactorArgs& a, const PanelItem* items, int count) {
  k_potrf_diag<<<count, 256, 0, st>>>(a, items);
}

void launch_trsm_rows(cudaStream_t st, const FactorArgs& a, const PanelItem* items, int count) {
  k_trsm_rows<<<count, 128, 0, st>>>(a, items);
}

void launch_permute_in(cudaStream_t st, double* X, int64_t ldx, const double* B, int64_t ldb,
                       const int32_t* invp0, int n, int nrhs) {
  k_permute_in<<<grid_for((int64_t)n * nrhs, 256), 256, 0, st>>>(X, ldx, B, ldb, invp0, n, nrhs);
}

void launch_permute_out(cudaStream_t st, double* B, int64_t ldb, const double* X, int64_t ldx,
                        const int32_t* invp0, int n, int nrhs) {
  k_permute_out<<<grid_for((int64_t)n * nrhs, 256), 256, 0, st>>>(B, ldb, X, ldx, invp0, n, nrhs);
}

}  // namespace dev
}  // namespace spb
