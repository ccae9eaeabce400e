// Supernodal Cholesky factor and solve kernels for sm_100a.
//
// Numerics follow symPACK's blockCell_t operations (symPACKMatrix2D.hpp):
//   factorize   1052-1102  Potrf of the diagonal block
//   trsm        1104-1178  L_KI = A_KI * L_II^-T
//   update      1180-1469  target(K,J) -= L_KI * L_JI^T, scattered through row/column maps
//   forward_update / forward_update_contrib   1486-1643
//   back_update / _tri_solve / back_update_contrib   1645-1797
// on a column-major panel per supernode instead of row-major cells.
// LDL^T (blockCellLDL_t, 2D.hpp:1802-2465): Potrf_LDL of the diagonal block
// (lapack.hpp:206-560, no pivoting, a zero pivot is reported), unit TRSM then
// scaling by 1/D (2D.hpp:2118-2137), updates with L D as the second operand
// (computeDLT, 2D.hpp:2140-2160).
#include <cfloat>
#include <climits>
#include <cstdio>

#include "factor_tasks.cuh"

namespace spb {
namespace dev {

namespace {

using namespace ftask;

template <class T>
__global__ void k_assemble(T* __restrict__ L, const int64_t* __restrict__ dst, const double* __restrict__ vals,
                           int64_t nnz) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x)
    L[dst[i]] = (T)vals[i];
}

template <class T>
__global__ void __launch_bounds__(128) k_factor_small(FactorArgs a, const int32_t* __restrict__ items) {
  extern __shared__ double sm_small[];
  factor_small_task<T>(a, items[blockIdx.x], sm_small);
}

template <class T>
__global__ void __launch_bounds__(kThreads, 1) k_potrf_diag(FactorArgs a, const PanelItem* __restrict__ items,
                                                         double* __restrict__ winv) {
  extern __shared__ double sm_diag[];
  potrf_diag_task<T>(a, items[blockIdx.x], winv, sm_diag);
}

template <class T>
__global__ void __launch_bounds__(kThreads, 1) k_ldl_diag(FactorArgs a, const PanelItem* __restrict__ items,
                                                       double* __restrict__ winv) {
  extern __shared__ double sm_ldl[];
  ldl_diag_task<T>(a, items[blockIdx.x], winv, sm_ldl);
}

template <class T>
__global__ void __launch_bounds__(kThreads, 2) k_trsm_rows(FactorArgs a, const PanelItem* __restrict__ items,
                                                        const double* __restrict__ winv) {
  extern __shared__ double sm_trsm[];
  trsm_rows_task<T>(a, items[blockIdx.x], winv, sm_trsm);
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
  for (auto f : {k_trsm_rows<double>, k_trsm_rows<float>})
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrsmSmemDoubles * (int)sizeof(double));
  for (auto f : {k_factor_small<double>, k_factor_small<float>})
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
  init_gemm_attributes();
  init_solve_attributes();
}

void launch_assemble(cudaStream_t st, void* L, bool fp32, const int64_t* dst, const double* vals, int64_t nnz) {
  if (nnz <= 0) return;
  if (fp32) k_assemble<float><<<grid_for(nnz, 256), 256, 0, st>>>(static_cast<float*>(L), dst, vals, nnz);
  else k_assemble<double><<<grid_for(nnz, 256), 256, 0, st>>>(static_cast<double*>(L), dst, vals, nnz);
}

void launch_factor_small(cudaStream_t st, const FactorArgs& a, const int32_t* items, int count, int smem_bytes) {
  if (a.fp32) k_factor_small<float><<<count, 128, smem_bytes, st>>>(a, items);
  else k_factor_small<double><<<count, 128, smem_bytes, st>>>(a, items);
}

void launch_potrf_diag(cudaStream_t st, const FactorArgs& a, const PanelItem* items, int count, double* winv) {
  const size_t smem = kDiagSmemDoubles * sizeof(double);
  if (a.ldl) k_ldl_diag<double><<<count, kThreads, smem, st>>>(a, items, winv);  // LDL^T is FP64 only
  else if (a.fp32) k_potrf_diag<float><<<count, kThreads, smem, st>>>(a, items, winv);
  else k_potrf_diag<double><<<count, kThreads, smem, st>>>(a, items, winv);
}

void launch_trsm_rows(cudaStream_t st, const FactorArgs& a, const PanelItem* items, int count, const double* winv) {
  const size_t smem = kTrsmSmemDoubles * sizeof(double);
  if (a.fp32) k_trsm_rows<float><<<count, kThreads, smem, st>>>(a, items, winv);
  else k_trsm_rows<double><<<count, kThreads, smem, st>>>(a, items, winv);
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
