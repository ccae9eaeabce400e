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

// TRSM of one 64-row tile below a factored diagonal block: R <- R D^-T.
__global__ void __launch_bounds__(256) k_trsm_rows(FactorArgs a, const PanelItem* __restrict__ items) {
  extern __shared__ double smem_tr[];
  double* D = smem_tr;
  double* R = smem_tr + kNB * kNB;
  const PanelItem it = items[blockIdx.x];
  const SnMeta m = a.meta[it.s];
  double* g = a.L + m.off;
  const int nb = it.nb, c0 = it.c0;
  const int64_t ld = m.ld;
  const int rows = min(64, m.h - it.row0);
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    int c = idx / nb, r = idx - c * nb;
    D[r + c * kNB] = (r >= c) ? g[(c0 + r) + (int64_t)(c0 + c) * ld] : 0.0;
  }
  for (int idx = threadIdx.x; idx < rows * nb; idx += blockDim.x) {
    int c = idx / rows, r = idx - c * rows;
    R[r + c * kNB] = g[(it.row0 + r) + (int64_t)(c0 + c) * ld];
  }
  __syncthreads();
  for (int k = 0; k < nb; ++k) {
    const double inv = 1.0 / D[k + k * kNB];
    for (int r = threadIdx.x; r < rows; r += blockDim.x) R[r + k * kNB] *= inv;
    __syncthreads();
    const int rem = nb - k - 1;
    for (int idx = threadIdx.x; idx < rows * rem; idx += blockDim.x) {
      int j = k + 1 + idx / rows, r = idx % rows;
      R[r + j * kNB] -= R[r + k * kNB] * D[j + k * kNB];
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < rows * nb; idx += blockDim.x) {
    int c = idx / rows, r = idx - c * rows;
    g[(it.row0 + r) + (int64_t)(c0 + c) * ld] = R[r + c * kNB];
  }
}

// Position of global row `row` in a sorted row list of length h, or -1.
__device__ __forceinline__ int find_row(const int32_t* __restrict__ rl, int h, int row) {
  int lo = 0, hi = h;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (rl[mid] < row) lo = mid + 1;
    else hi = mid;
  }
  return (lo < h && rl[lo] == row) ? lo : -1;
}

// 64 x 64 tile of C = A B^T (FP64), 256 threads holding 4 x 4 each.
__global__ void __launch_bounds__(256) k_gemm64(FactorArgs a, const TileItem* __restrict__ items) {
  __shared__ double As[16][64];
  __shared__ double Bs[16][64];
  __shared__ int Rr[64], Rc[64], Tc[64], Pos[64];
  const TileItem it = items[blockIdx.x];
  const SnMeta m = a.meta[it.s];
  double* g = a.L + m.off;
  const int64_t ld = m.ld;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;

  for (int kk = 0; kk < it.kn; kk += 16) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int e = tid + 256 * q, kq = e >> 6, r = e & 63, k = kk + kq;
      const int64_t col = (int64_t)(it.k0 + k) * ld;
      As[kq][r] = (r < it.mrows && k < it.kn) ? g[it.a_row0 + r + col] : 0.0;
      Bs[kq][r] = (r < it.ncols && k < it.kn) ? g[it.b_row0 + r + col] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kq = 0; kq < 16; ++kq) {
      double av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kq][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kq][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
    __syncthreads();
  }

  if (it.mode == 0) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int r = ty + 16 * i, c = tx + 16 * j;
        if (r < it.mrows && c < it.ncols) {
          int gr = it.a_row0 + r, gc = it.b_row0 + c;
          if (gr >= gc) g[gr + (int64_t)gc * ld] -= acc[i][j];
        }
      }
    return;
  }
  // scatter-subtract into the ancestors owning rows Rr x columns Rc
  const int32_t* rl = a.rows + m.lidx;
  if (tid < 64) {
    Rr[tid] = tid < it.mrows ? rl[it.a_row0 + tid] : INT_MAX;
    int rc = tid < it.ncols ? rl[it.b_row0 + tid] : INT_MAX;
    Rc[tid] = rc;
    Tc[tid] = tid < it.ncols ? a.supmember[rc] : -1;
  }
  __syncthreads();
  int c = 0;
  while (c < it.ncols) {
    const int t = Tc[c];
    int ce = c + 1;
    while (ce < it.ncols && Tc[ce] == t) ++ce;
    const SnMeta mt = a.meta[t];
    if (tid < 64) {
      int pos = -1;
      if (tid < it.mrows && Rr[tid] >= Rc[c]) {
        pos = find_row(a.rows + mt.lidx, mt.h, Rr[tid]);
        if (pos < 0) report(a.status, 2, it.s, Rr[tid]);
      }
      Pos[tid] = pos;
    }
    __syncthreads();
    double* gt = a.L + mt.off;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int r = ty + 16 * i, cc = tx + 16 * j;
        if (cc >= c && cc < ce && r < it.mrows && Rr[r] >= Rc[cc]) {
          int p = Pos[r];
          if (p >= 0) atomicAdd(gt + (int64_t)(Rc[cc] - mt.fc) * mt.ld + p, -acc[i][j]);
        }
      }
    __syncthreads();
    c = ce;
  }
}

// ---------------------------------------------------------------- solve ----

// Forward substitution for one supernode: Y_J <- L_JJ^-1 Y_J, then
// Y_K[rows] -= L_KJ Y_J (2D.hpp:1519-1527, 1589-1592), blocked by 64 columns.
__global__ void __launch_bounds__(256) k_solve_fwd(SolveArgs a, const int32_t* __restrict__ sn) {
  __shared__ double Y[64 * 64];
  const int s = sn[blockIdx.x];
  const SnMeta m = a.meta[s];
  const double* P = a.L + m.off;
  const int32_t* rl = a.rows + m.lidx;
  const int64_t ld = m.ld;
  const int nrhs = a.nrhs;
  for (int cb = 0; cb < m.w; cb += 64) {
    const int nb = min(64, m.w - cb);
    for (int idx = threadIdx.x; idx < nb * nrhs; idx += blockDim.x) {
      int c = idx / nb, k = idx - c * nb;
      Y[k + c * 64] = a.X[(m.fc + cb + k) + c * a.ldx];
    }
    __syncthreads();
    for (int k = 0; k < nb; ++k) {
      const double inv = 1.0 / P[(cb + k) + (int64_t)(cb + k) * ld];
      for (int c = threadIdx.x; c < nrhs; c += blockDim.x) Y[k + c * 64] *= inv;
      __syncthreads();
      const int rem = nb - k - 1;
      for (int idx = threadIdx.x; idx < rem * nrhs; idx += blockDim.x) {
        int c = idx / rem, j = k + 1 + (idx - c * rem);
        Y[j + c * 64] -= P[(cb + j) + (int64_t)(cb + k) * ld] * Y[k + c * 64];
      }
      __syncthreads();
    }
    for (int idx = threadIdx.x; idx < nb * nrhs; idx += blockDim.x) {
      int c = idx / nb, k = idx - c * nb;
      a.X[(m.fc + cb + k) + c * a.ldx] = Y[k + c * 64];
    }
    const int r0 = cb + nb, rows = m.h - r0;
    for (int idx = threadIdx.x; idx < rows * nrhs; idx += blockDim.x) {
      int c = idx / rows, r = r0 + (idx - c * rows);
      double sum = 0.0;
      for (int k = 0; k < nb; ++k) sum = fma(P[r + (int64_t)(cb + k) * ld], Y[k + c * 64], sum);
      if (r < m.w) a.X[(m.fc + r) + c * a.ldx] -= sum;
      else atomicAdd(&a.X[rl[r] + c * a.ldx], -sum);
    }
    __syncthreads();
  }
}

// Backward substitution for one supernode: X_J -= L_KJ^T X_K[rows], then
// X_J <- L_JJ^-T X_J (2D.hpp:1659-1721, 1741-1744), blocked by 64 columns.
__global__ void __launch_bounds__(256) k_solve_bwd(SolveArgs a, const int32_t* __restrict__ sn) {
  __shared__ double Z[64 * 64];
  const int s = sn[blockIdx.x];
  const SnMeta m = a.meta[s];
  const double* P = a.L + m.off;
  const int32_t* rl = a.rows + m.lidx;
  const int64_t ld = m.ld;
  const int nrhs = a.nrhs;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int lastcb = ((m.w - 1) / 64) * 64;
  for (int cb = lastcb; cb >= 0; cb -= 64) {
    const int nb = min(64, m.w - cb);
    const int r0 = cb + nb;
    for (int pair = warp; pair < nb * nrhs; pair += nw) {
      int c = pair / nb, k = pair - c * nb;
      double sum = 0.0;
      for (int r = r0 + lane; r < m.h; r += 32) {
        int grow = r < m.w ? m.fc + r : rl[r];
        sum = fma(P[r + (int64_t)(cb + k) * ld], a.X[grow + c * a.ldx], sum);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      if (lane == 0) Z[k + c * 64] = a.X[(m.fc + cb + k) + c * a.ldx] - sum;
    }
    __syncthreads();
    for (int k = nb - 1; k >= 0; --k) {
      const double inv = 1.0 / P[(cb + k) + (int64_t)(cb + k) * ld];
      for (int c = threadIdx.x; c < nrhs; c += blockDim.x) Z[k + c * 64] *= inv;
      __syncthreads();
      for (int idx = threadIdx.x; idx < k * nrhs; idx += blockDim.x) {
        int c = idx / k, j = idx - c * k;
        Z[j + c * 64] -= P[(cb + k) + (int64_t)(cb + j) * ld] * Z[k + c * 64];
      }
      __syncthreads();
    }
    for (int idx = threadIdx.x; idx < nb * nrhs; idx += blockDim.x) {
      int c = idx / nb, k = idx - c * nb;
      a.X[(m.fc + cb + k) + c * a.ldx] = Z[k + c * 64];
    }
    __syncthreads();
  }
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
  cudaFuncSetAttribute(k_factor_small, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
  cudaFuncSetAttribute(k_trsm_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * kNB * kNB * sizeof(double));
}

void launch_factor_small(cudaStream_t st, const FactorArgs& a, const int32_t* items, int count, int smem_bytes) {
  k_factor_small<<<count, 128, smem_bytes, st>>>(a, items);
}

void launch_potrf_diag(cudaStream_t st, const FactorArgs& a, const PanelItem* items, int count) {
  k_potrf_diag<<<count, 256, 0, st>>>(a, items);
}

void launch_trsm_rows(cudaStream_t st, const FactorArgs& a, const PanelItem* items, int count) {
  k_trsm_rows<<<count, 256, 2 * kNB * kNB * sizeof(double), st>>>(a, items);
}

void launch_gemm(cudaStream_t st, const FactorArgs& a, const TileItem* items, int count, int tile) {
  (void)tile;
  k_gemm64<<<count, 256, 0, st>>>(a, items);
}

void launch_solve_forward(cudaStream_t st, const SolveArgs& a, const int32_t* sn, int count) {
  k_solve_fwd<<<count, 256, 0, st>>>(a, sn);
}

void launch_solve_backward(cudaStream_t st, const SolveArgs& a, const int32_t* sn, int count) {
  k_solve_bwd<<<count, 256, 0, st>>>(a, sn);
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
