// FP64 iterative refinement around an FP32 factor (precision form).
//
// Each step computes r = b - A x with the original matrix in FP64, measures the
// backward error eta = ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) per
// right-hand side and per system (a batch of block-diagonal systems is measured
// system by system, with that system's own norms), solves A d = r with the FP32 factor and updates x += d in FP64.
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

// Per-system maxima.  Rows are grouped into systems (segments) given by
// rowseg[i] (nullptr: one system); out[seg * 64 + c] = max |v[i + c*ld]| over
// the rows i of that system.  Each CTA takes a contiguous chunk of rows, each
// thread keeps a running maximum while its rows stay in one system, and a warp
// whose lanes end in the same system merges before the atomic.  out zeroed by
// the caller.
constexpr int kChunk = 4096;

__device__ __forceinline__ void flush_segmax(double* out, int seg, double m) {
  const unsigned full = 0xffffffffu;
  const int seg0 = __shfl_sync(full, seg, 0);
  if (__all_sync(full, seg == seg0)) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(full, m, o));
    if ((threadIdx.x & 31) == 0 && seg0 >= 0) atomic_max_nonneg(out + seg0 * 64, m);
  } else if (seg >= 0) {
    atomic_max_nonneg(out + seg * 64, m);
  }
}

__global__ void k_segmax(const double* __restrict__ v, int n, int nrhs, int64_t ld, const int32_t* __restrict__ rowseg,
                         double* __restrict__ out) {
  const int64_t r0 = (int64_t)blockIdx.x * kChunk;
  const int64_t r1 = min((int64_t)n, r0 + kChunk);
  for (int c = 0; c < nrhs; ++c) {
    int seg = -1;
    double m = 0.0;
    for (int64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      const int si = rowseg ? rowseg[i] : 0;
      if (si != seg) {
        if (seg >= 0) atomic_max_nonneg(out + seg * 64 + c, m);
        seg = si;
        m = 0.0;
      }
      m = fmax(m, fabs(v[i + c * ld]));
    }
    flush_segmax(out + c, seg, m);
  }
}

// anorm[seg] = max over the rows i of the system of sum_j |A_ij|
__global__ void k_rowsum_segmax(const int64_t* __restrict__ rowptr, const double* __restrict__ val, int n,
                                const int32_t* __restrict__ rowseg, double* __restrict__ anorm) {
  const int64_t r0 = (int64_t)blockIdx.x * kChunk;
  const int64_t r1 = min((int64_t)n, r0 + kChunk);
  int seg = -1;
  double m = 0.0;
  for (int64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const int si = rowseg ? rowseg[i] : 0;
    if (si != seg) {
      if (seg >= 0) atomic_max_nonneg(anorm + seg, m);
      seg = si;
      m = 0.0;
    }
    double s = 0.0;
    for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p) s += fabs(val[p]);
    m = fmax(m, s);
  }
  const unsigned full = 0xffffffffu;
  const int seg0 = __shfl_sync(full, seg, 0);
  if (__all_sync(full, seg == seg0)) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(full, m, o));
    if ((threadIdx.x & 31) == 0 && seg0 >= 0) atomic_max_nonneg(anorm + seg0, m);
  } else if (seg >= 0) {
    atomic_max_nonneg(anorm + seg, m);
  }
}

// eta = max over systems and right-hand sides of rmax / (anorm * xmax + bmax):
// the normwise backward error of every system by itself.
__global__ void k_eta(const double* __restrict__ anorm, const double* __restrict__ bmax,
                      const double* __restrict__ xmax, const double* __restrict__ rmax, int nseg, int nrhs,
                      double* __restrict__ eta) {
  double e = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nseg * nrhs; k += gridDim.x * blockDim.x) {
    const int seg = k / nrhs, c = k - seg * nrhs;
    const double r = rmax[seg * 64 + c];
    const double den = anorm[seg] * xmax[seg * 64 + c] + bmax[seg * 64 + c];
    e = fmax(e, den > 0.0 ? r / den : (r > 0.0 ? 1e300 : 0.0));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(eta, e);
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

void launch_segmax(cudaStream_t st, const double* v, int n, int nrhs, int64_t ld, const int32_t* rowseg,
                   double* out) {
  k_segmax<<<(n + kChunk - 1) / kChunk, 256, 0, st>>>(v, n, nrhs, ld, rowseg, out);
}

void launch_rowsum_segmax(cudaStream_t st, const int64_t* rowptr, const double* val, int n, const int32_t* rowseg,
                          double* anorm) {
  k_rowsum_segmax<<<(n + kChunk - 1) / kChunk, 256, 0, st>>>(rowptr, val, n, rowseg, anorm);
}

void launch_eta(cudaStream_t st, const double* anorm, const double* bmax, const double* xmax, const double* rmax,
                int nseg, int nrhs, double* eta) {
  k_eta<<<grid_for((int64_t)nseg * nrhs, 256), 256, 0, st>>>(anorm, bmax, xmax, rmax, nseg, nrhs, eta);
}

void launch_axpy(cudaStream_t st, double* x, const double* d, int n, int nrhs, int64_t ld) {
  k_axpy<<<grid_for((int64_t)n * nrhs, 256), 256, 0, st>>>(x, d, n, nrhs, ld);
}

}  // namespace dev
}  // namespace spb
