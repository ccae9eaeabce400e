// FP64 iterative refinement around an FP32 factor (precision form).
//
// Each step computes r = b - A x with the original matrix in FP64, measures the
// backward error eta = ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) per
// right-hand side, solves A d = r with the FP32 factor and updates x += d in FP64.
// A is held as full symmetric CSR in the original ordering; its values are
// gathered from the lower-triangle input on every DistributeMatrix.
#include "kernels.cuh"

namespace spb {
namespace dev {

namespace {

int grid_for(int64_t work, int threads) {
  int64_t g = (work + threads - 1) / threads;
  if (g > 148 * 16) g = 148 * 16;
  return g < 1 ? 1 : (int)g;
}

__global__ void k_gather(double* __restrict__ dst, const double* __restrict__ src, const int64_t* __restrict__ idx,
                         int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[idx[i]];
}

// Non-negative doubles order like their bit patterns: max through 64-bit integer atomics.
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// r = b - A x, one warp per row and right-hand side column.
__global__ void k_residual(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                           const double* __restrict__ val, const double* __restrict__ x, const double* __restrict__ b,
                           double* __restrict__ r, int n, int nrhs, int64_t ld) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t w = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); w < (int64_t)n * nrhs; w += warps) {
    const int c = (int)(w / n), i = (int)(w - (int64_t)c * n);
    const double* xc = x + c * ld;
    double s = 0.0;
    for (int64_t p = rowptr[i] + lane; p < rowptr[i + 1]; p += 32) s = fma(val[p], xc[col[p]], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) r[i + c * ld] = b[i + c * ld] - s;
  }
}

// out[c] = max_i |v[i + c*ld]|  (out zeroed by the caller)
__global__ void k_colmax(const double* __restrict__ v, int n, int nrhs, int64_t ld, double* __restrict__ out) {
  for (int c = 0; c < nrhs; ++c) {
    double m = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      m = fmax(m, fabs(v[i + c * ld]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out + c, m);
  }
}

// out = max_i sum_j |A_ij|
__global__ void k_rowsum_max(const int64_t* __restrict__ rowptr, const double* __restrict__ val, int n,
                             double* __restrict__ out) {
  double m = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p) s += fabs(val[p]);
    m = fmax(m, s);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, m);
}

__global__ void k_axpy(double* __restrict__ x, const double* __restrict__ d, int n, int nrhs, int64_t ld) {
  const int64_t total = (int64_t)n * nrhs;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(k / n), i = (int)(k - (int64_t)c * n);
    x[i + c * ld] += d[i + c * ld];
  }
}

}  // namespace

void launch_gather(cudaStream_t st, double* dst, const double* src, const int64_t* idx, int64_t n) {
  if (n > 0) k_gather<<<grid_for(n, 256), 256, 0, st>>>(dst, src, idx, n);
}

void launch_residual(cudaStream_t st, const int64_t* rowptr, const int32_t* col, const double* val, const double* x,
                     const double* b, double* r, int n, int nrhs, int64_t ld) {
  k_residual<<<grid_for((int64_t)n * nrhs * 32, 256), 256, 0, st>>>(rowptr, col, val, x, b, r, n, nrhs, ld);
}

void launch_colmax(cudaStream_t st, const double* v, int n, int nrhs, int64_t ld, double* out) {
  k_colmax<<<grid_for(n, 256), 256, 0, st>>>(v, n, nrhs, ld, out);
}

void launch_rowsum_max(cudaStream_t st, const int64_t* rowptr, const double* val, int n, double* out) {
  k_rowsum_max<<<grid_for(n, 256), 256, 0, st>>>(rowptr, val, n, out);
}

void launch_axpy(cudaStream_t st, double* x, const double* d, int n, int nrhs, int64_t ld) {
  k_axpy<<<grid_for((int64_t)n * nrhs, 256), 256, 0, st>>>(x, d, n, nrhs, ld);
}

}  // namespace dev
}  // namespace spb
