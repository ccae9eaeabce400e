// Schur-complement products of the supernodal factorization (sm_100a):
//   C = A * B^T over panel columns [k0, k0 + kn) of one supernode, followed by
//   either an in-panel subtraction (mode 0) or a scatter-subtraction into the
//   ancestor panels that own the rows and columns of C (mode 1).  This is the
//   blockCell_t::update of symPACKMatrix2D.hpp:1180-1469 (GEMM into a buffer,
//   then the src_to_tgt_offset / colindx scatter of 2D.hpp:1395-1466), fused so
//   that C never leaves the SM.
//
// Tile engines (one shared epilogue for the tiles staged in shared memory):
//   k_gemm_dmma   128 x 64 FP64 tiles on the FP64 tensor pipe (mma.sync m16n8k4 .f64),
//                 3-stage cp.async pipeline, 8 warps of 32 x 32, two CTAs per SM
//   k_gemm_simt   64 x 64 tiles with FMA, for narrow updates
//   k_gemm_tc32   128 x 128 FP32 tiles, 3xTF32 on tcgen05, operands staged by cp.async
//   k_gemm_tc32w  the same on TMA-loaded split copies, persistent and warp-specialised
//                 (tc32t_tile_task: one such tile, a task of the persistent FP32 factorization)
//   k_gemm_tc32p, k_gemm_tf32x3   a persistent tcgen05 variant and an mma.sync one
// The epilogue stages C in shared memory and walks it column by column, so
// consecutive threads touch consecutive target rows (coalesced atomics).
#include <climits>
#include <type_traits>

#include "factor_tasks.cuh"

namespace spb {
namespace dev {

namespace {

__device__ __forceinline__ void report_status(Status* st, int code, int s, int col) {
  if (atomicCAS(&st->code, 0, code) == 0) {
    st->supernode = s;
    st->column = col;
  }
}

// Apply a BM x BN tile of C held in shared memory (column-major, leading dimension ldc),
// subtracting it with fire-and-forget atomic reductions (no load on the thread's
// critical path).  Each thread keeps one tile row (consecutive threads take
// consecutive rows, so the reductions of a warp are coalesced) and walks the
// columns.  Mode 1 targets come from the relative indices computed with the plan:
// per tile column its target column base and group offset (staged in shared
// memory); the row's position in a target is loaded once per target group, since
// the columns of one group share it.
template <int BM, int BN, int NT, class T, class CT>
__device__ void tile_epilogue(const FactorArgs& a, const TileItem& it, const SnMeta& m, const CT* Cs, int ldc,
                              int64_t* Cbase, int64_t* Crel) {
  static_assert(NT % BM == 0, "one row per thread");
  const int tid = threadIdx.x, i = tid % BM, c0 = tid / BM;
  constexpr int kStep = NT / BM;
  T* L = static_cast<T*>(a.L);
  const int jr = it.a_row0 + i;
  if (it.mode == 0) {
    if constexpr (std::is_same<T, float>::value && std::is_same<CT, float>::value && BM % 128 == 0) {
      // FP32 panel: 4 consecutive rows per thread and one 16-byte vector reduction per
      // column; panels start on 32-element boundaries, leading dimensions are multiples
      // of 4 and in-panel tiles start on 64-row boundaries, so the 4 rows are aligned
      const int q4 = tid % (BM / 4), cp = tid / (BM / 4), i0 = 4 * q4;
      constexpr int kCStep = NT / (BM / 4);
      const int jr0 = it.a_row0 + i0;
      T* g = L + m.off + jr0;
      for (int c = cp; c < it.ncols; c += kCStep) {
        const int gc = it.b_row0 + c;
        const float4 v = *reinterpret_cast<const float4*>(Cs + i0 + c * ldc);
        if (i0 + 3 < it.mrows && jr0 >= gc) {
          atomicAdd(reinterpret_cast<float4*>(g + (int64_t)gc * m.ld), make_float4(-v.x, -v.y, -v.z, -v.w));
        } else {
          const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (i0 + e < it.mrows && jr0 + e >= gc) atomicAdd(g + e + (int64_t)gc * m.ld, -vv[e]);
        }
      }
      return;
    }
    if (i >= it.mrows) return;
    T* g = L + m.off + jr;
    for (int c = c0; c < it.ncols; c += kStep) {
      const int gc = it.b_row0 + c;
      if (jr >= gc) atomicAdd(g + (int64_t)gc * m.ld, (T)(-Cs[i + c * ldc]));
    }
    return;
  }
  const int32_t* rl = a.rows + m.lidx;
  for (int c = tid; c < BN; c += NT) {
    if (c < it.ncols) {
      const int jc = it.b_row0 + c;
      const RelGroup g = a.groups[a.row_group[m.lidx + jc]];
      const SnMeta mt = a.meta[g.t];
      Cbase[c] = mt.off + (int64_t)(rl[jc] - mt.fc) * mt.ld;
      Crel[c] = g.rel_off - g.j0;
    }
  }
  __syncthreads();
  if (i >= it.mrows) return;
  int64_t last = INT64_MIN;  // group offsets (rel_off - j0) can be negative
  int pos = 0;
  for (int c = c0; c < it.ncols; c += kStep) {
    if (jr < it.b_row0 + c) break;  // rows are sorted: later columns are above this row
    const int64_t cr = Crel[c];
    if (cr != last) {
      pos = a.rel[cr + jr];
      last = cr;
    }
    atomicAdd(L + Cbase[c] + pos, (T)(-Cs[i + c * ldc]));
  }
}

}  // namespace

namespace {

// Bounded wait for the phase of an mbarrier with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
  for (long long i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.b32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// ---- 128 x BN FP64 tensor-core tile ------------------------------------------------
// BN = 64: 8 warps of 32 x 32 (4 x 2), two CTAs per SM (126 registers, 102 KB of shared
// memory each), so that one CTA's prologue and atomic epilogue overlap the other's MMAs.
// Operands arrive by bulk asynchronous copies (cp.async.bulk, the TMA engine's untiled
// form): per 16-column stage one copy per panel column and operand (128 or BN rows, 1 KB /
// 512 B) into a padded column-major layout whose fragment reads are bank-conflict free,
// issued by the lanes of warp 0 and completed on the stage's mbarrier (transaction bytes);
// every warp releases a stage on a second mbarrier once it has read it, and warp 0
// refills it.  No block-wide barrier in the K loop.  Copies start on 16-byte boundaries,
// so an operand's rows are counted from the even row at or below its first row: accumulator
// row i is panel row (a_row0 & ~1) + i (the plan cuts these tiles so that they fit).
constexpr int kDM = 128, kDK = 16, kDStages = 4, kDLds = 132, kDLdc = 130, kDThreads = 256;
constexpr int kDTileN = 64;  // FP64 update tiles are 128 x 64
template <int BN>
struct DTile {
  static constexpr int kLdb = BN + 4;
  static constexpr int kWarpsN = BN / 32, kWarpsM = 8 / kWarpsN;
  static constexpr int kMI = kDM / kWarpsM / 16;  // 16-row MMA tiles per warp
  static constexpr int kStageElems = kDK * (kDLds + kLdb);
  static constexpr size_t kPipeBytes = (size_t)kDStages * kStageElems * sizeof(double);
  static constexpr size_t kCBytes = (size_t)BN * kDLdc * sizeof(double);
  static constexpr size_t kMainBytes = kPipeBytes > kCBytes ? kPipeBytes : kCBytes;
  static constexpr size_t kIntsBytes = 4 * 128 * sizeof(int);
  static constexpr size_t kSmemBytes = kMainBytes + kIntsBytes + 2 * kDStages * sizeof(uint64_t);
  static_assert((kDLds * 8) % 16 == 0 && (kLdb * 8) % 16 == 0 && (kStageElems * 8) % 16 == 0,
                "bulk copy destinations on 16-byte boundaries");
};
constexpr size_t kDSmemBytes = DTile<kDTileN>::kSmemBytes;

// D = A(16x4, row) * B(4x8, col) + D, FP64.  Fragment ownership (lane = 4*g + t):
//   a0 = A[g][t], a1 = A[g+8][t], b0 = B[t][g],
//   d0 = D[g][2t], d1 = D[g][2t+1], d2 = D[g+8][2t], d3 = D[g+8][2t+1].
__device__ __forceinline__ void dmma_16x8x4(double* d, double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

constexpr long long kDWaitLimit = 1LL << 24;  // mbarrier polls before a DMMA tile gives up (seconds)
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// Stage barriers of the DMMA tile, kept across the tiles a persistent CTA runs: g counts the
// stages this CTA has consumed, so stage q of its life uses buffer q % kDStages and phase
// (q / kDStages) & 1 of that buffer's barriers.
struct DmPipe {
  uint64_t* full;   // copies landed: one arrival (with the byte count) + transaction bytes
  uint64_t* empty;  // read by all 8 warps
  uint32_t g;
};

template <int BN>
__device__ __forceinline__ void dm_setup(DmPipe& P, unsigned char* smem_raw) {
  using D = DTile<BN>;
  P.full = reinterpret_cast<uint64_t*>(smem_raw + D::kMainBytes + D::kIntsBytes);
  P.empty = P.full + kDStages;
  P.g = 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kDStages; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(P.full + i)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(P.empty + i)), "r"(kDThreads / 32)
                   : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
}

// One 128 x BN DMMA tile (kDThreads threads, DTile<BN>::kSmemBytes of shared memory).
// Returns false, after recording status 3, when a barrier wait gave up (the copies in
// flight have then been waited for, bounded).
template <int BN>
__device__ bool dmma_tile_task(const FactorArgs& a, const TileItem& it, unsigned char* smem_raw, DmPipe& P) {
  using D = DTile<BN>;
  __shared__ int sh_abort;
  double* pipe = reinterpret_cast<double*>(smem_raw);
  double* Cs = reinterpret_cast<double*>(smem_raw);  // reused once the main loop is done
  int* ints = reinterpret_cast<int*>(smem_raw + D::kMainBytes);
  const SnMeta m = a.meta[it.s];
  const double* g = static_cast<const double*>(a.L) + m.off;
  const double* gb = a.ldl ? a.W + m.off : g;  // second operand: L, or L D for LDL^T
  const int64_t ld = m.ld;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % D::kWarpsM, wn = warp / D::kWarpsM;
  const int gq = lane >> 2, tq = lane & 3;
  const int a0 = it.a_row0 & ~1, b0 = it.b_row0 & ~1;
  const int ashift = it.a_row0 - a0, bshift = it.b_row0 - b0;
  // rows copied per column: the tile's rows, within the column's padded storage (ld, a
  // multiple of 4, so the count is even and the copy a multiple of 16 bytes)
  const int nra = (int)min((int64_t)kDM, ld - a0), nrb = (int)min((int64_t)BN, ld - b0);
  const int nk = (it.kn + kDK - 1) / kDK;
  const uint32_t g0 = P.g;

  // earlier generic-proxy accesses of the stages (other tasks, the last epilogue) come
  // before this tile's copies
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (tid == 0) sh_abort = 0;
  __syncthreads();

  // stage kt (all lanes of warp 0): zero the K lines past kn up to the next multiple of 4,
  // then one column copy per lane (A: lanes 0-15, B: lanes 16-31)
  int issued = 0;
  auto issue = [&](int kt) {
    const uint32_t q = g0 + kt;
    double* As = pipe + (size_t)(q % kDStages) * D::kStageElems;
    double* Bs = As + kDK * kDLds;
    const int kv = min(kDK, it.kn - kt * kDK), kz = min(kDK, (kv + 3) & ~3);
    for (int e = lane; e < (kz - kv) * (kDLds + D::kLdb); e += 32) {
      const int l = kv + e / (kDLds + D::kLdb), o = e % (kDLds + D::kLdb);
      if (o < kDLds) As[l * kDLds + o] = 0.0;
      else Bs[l * D::kLdb + o - kDLds] = 0.0;
    }
    const uint32_t bar = smem_u32(P.full + q % kDStages);
    __syncwarp();
    if (lane == 0)
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar),
                   "r"((uint32_t)(kv * (nra + nrb) * 8))
                   : "memory");
    __syncwarp();
    const int64_t k = it.k0 + (int64_t)kt * kDK;
    if (lane < kv) bulk_g2s(smem_u32(As + lane * kDLds), g + a0 + (k + lane) * ld, (uint32_t)nra * 8, bar);
    else if (lane >= 16 && lane - 16 < kv)
      bulk_g2s(smem_u32(Bs + (lane - 16) * D::kLdb), gb + b0 + (k + lane - 16) * ld, (uint32_t)nrb * 8, bar);
    ++issued;
  };
  if (warp == 0)
    for (int kt = 0; kt < nk && kt < kDStages; ++kt) issue(kt);

  double acc[D::kMI][4][4];
#pragma unroll
  for (int i = 0; i < D::kMI; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;

  bool ok = true;
  for (int kt = 0; kt < nk; ++kt) {
    const uint32_t q = g0 + kt;
    const int st = q % kDStages;
    if (!mbar_wait(smem_u32(P.full + st), (q / kDStages) & 1, kDWaitLimit)) {
      ok = false;
      break;
    }
    const double* As = pipe + (size_t)st * D::kStageElems;
    const double* Bs = As + kDK * kDLds;
    const int kz = min(kDK, ((it.kn - kt * kDK) + 3) & ~3);
    // m16n8k4 steps: the B fragments of the warp's four column tiles, then per row tile
    // its A fragment and four MMAs
#pragma unroll
    for (int kk = 0; kk < kDK; kk += 4) {
      if (kk >= kz) break;
      double bf[4];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bf[ni] = Bs[(kk + tq) * D::kLdb + wn * 32 + ni * 8 + gq];
#pragma unroll
      for (int mi = 0; mi < D::kMI; ++mi) {
        const int r0 = wm * (16 * D::kMI) + mi * 16 + gq;
        const double x0 = As[(kk + tq) * kDLds + r0], x1 = As[(kk + tq) * kDLds + r0 + 8];
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma_16x8x4(acc[mi][ni], x0, x1, bf[ni]);
      }
    }
    __syncwarp();
    if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(P.empty + st)) : "memory");
    // warp 0 refills the buffer of the previous stage once every warp has read it
    const int pk = kt - 1;
    if (warp == 0 && pk >= 0 && pk + kDStages < nk) {
      const uint32_t pq = g0 + pk;
      if (!mbar_wait(smem_u32(P.empty + pq % kDStages), (pq / kDStages) & 1, kDWaitLimit)) {
        ok = false;
        break;
      }
      issue(pk + kDStages);
    }
  }
  if (!ok) sh_abort = 1;
  ok = __syncthreads_and(ok) != 0;
  if (!ok) {
    if (warp == 0 && lane == 0) {  // let this CTA's copies in flight land (bounded)
      for (int kt = 0; kt < issued; ++kt) {
        const uint32_t q = g0 + kt;
        mbar_wait(smem_u32(P.full + q % kDStages), (q / kDStages) & 1, kDWaitLimit);
      }
      report_status(a.status, 3, it.s, -1);
    }
    __syncthreads();
    P.g = g0 + nk;
    return false;
  }
  P.g = g0 + nk;
  // accumulator row r / column c are panel rows a0 + r / b0 + c; Cs holds the tile from
  // a_row0 / b_row0
#pragma unroll
  for (int mi = 0; mi < D::kMI; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
      const int r0 = wm * (16 * D::kMI) + mi * 16 + gq - ashift, c0 = wn * 32 + ni * 8 + 2 * tq - bshift;
      if (r0 >= 0 && c0 >= 0) Cs[r0 + c0 * kDLdc] = acc[mi][ni][0];
      if (r0 >= 0 && c0 + 1 >= 0) Cs[r0 + (c0 + 1) * kDLdc] = acc[mi][ni][1];
      if (c0 >= 0) Cs[r0 + 8 + c0 * kDLdc] = acc[mi][ni][2];
      if (c0 + 1 >= 0) Cs[r0 + 8 + (c0 + 1) * kDLdc] = acc[mi][ni][3];
    }
  __syncthreads();
  tile_epilogue<kDM, BN, kDThreads, double, double>(a, it, m, Cs, kDLdc, (int64_t*)ints, (int64_t*)ints + 128);
  return true;
}

__global__ void __launch_bounds__(kDThreads, 2) k_gemm_dmma(FactorArgs a, const TileItem* __restrict__ items) {
  extern __shared__ __align__(16) unsigned char smem_dmma[];
  DmPipe P;
  dm_setup<kDTileN>(P, smem_dmma);
  dmma_tile_task<kDTileN>(a, items[blockIdx.x], smem_dmma, P);
}

// ---- 64 x 64 FP64 FMA tile --------------------------------------------------------
constexpr int kSLdc = 65;
constexpr size_t kSCBytes = (size_t)64 * kSLdc * sizeof(double);
constexpr size_t kSSmemBytes = kSCBytes + 4 * 64 * sizeof(int);

// One 64 x 64 FMA tile (256 threads, kSSmemBytes of shared memory).
template <class T>
__device__ __noinline__ void simt_tile_task(const FactorArgs& a, const TileItem& it, unsigned char* smem_raw) {
  T(*As)[64] = reinterpret_cast<T(*)[64]>(smem_raw);
  T(*Bs)[64] = reinterpret_cast<T(*)[64]>(smem_raw + 16 * 64 * sizeof(T));
  T* Cs = reinterpret_cast<T*>(smem_raw);
  int* ints = reinterpret_cast<int*>(smem_raw + kSCBytes);
  const SnMeta m = a.meta[it.s];
  const T* g = static_cast<const T*>(a.L) + m.off;
  // second operand: L, or L D for LDL^T (FP64 only, so W is read only when T is double)
  const T* gb = a.ldl ? reinterpret_cast<const T*>(a.W + m.off) : g;
  const int64_t ld = m.ld;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
  for (int kk = 0; kk < it.kn; kk += 16) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int e = tid + 256 * q, kq = e >> 6, r = e & 63, k = kk + kq;
      const int64_t col = (int64_t)(it.k0 + k) * ld;
      As[kq][r] = (r < it.mrows && k < it.kn) ? g[it.a_row0 + r + col] : T(0);
      Bs[kq][r] = (r < it.ncols && k < it.kn) ? gb[it.b_row0 + r + col] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int kq = 0; kq < 16; ++kq) {
      T av[4], bv[4];
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
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) Cs[(ty + 16 * i) + (tx + 16 * j) * kSLdc] = acc[i][j];
  __syncthreads();
  tile_epilogue<64, 64, 256, T, T>(a, it, m, Cs, kSLdc, (int64_t*)ints, (int64_t*)ints + 64);
}

template <class T>
__global__ void __launch_bounds__(256) k_gemm_simt(FactorArgs a, const TileItem* __restrict__ items) {
  extern __shared__ __align__(16) unsigned char smem_simt[];
  simt_tile_task<T>(a, items[blockIdx.x], smem_simt);
}

// ---- 128 x 128 split-precision 3xTF32 tensor-core tile (FP32 storage) -------------
// Each FP32 operand x is split into tf32 parts hi = rna(x), lo = rna(x - hi);
// C += A_lo B_hi + A_hi B_lo + A_hi B_hi with FP32 accumulation, which recovers
// close to FP32 accuracy from the TF32 tensor pipe.
constexpr int kTK = 32, kTStages = 3, kTLds = 136, kTLdc = 132;
constexpr size_t kTPipeBytes = (size_t)kTStages * 2 * kTK * kTLds * sizeof(float);
constexpr size_t kTCBytes = (size_t)128 * kTLdc * sizeof(float);
constexpr size_t kTMainBytes = kTPipeBytes > kTCBytes ? kTPipeBytes : kTCBytes;
constexpr size_t kTSmemBytes = kTMainBytes + 4 * 128 * sizeof(int);

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes));
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

// D(16x8, f32) += A(16x8, tf32, row) * B(8x8, tf32, col); lane = 4*g + t:
//   a0 = A[g][t], a1 = A[g+8][t], a2 = A[g][t+4], a3 = A[g+8][t+4], b0 = B[t][g], b1 = B[t+4][g]
__device__ __forceinline__ void mma_tf32(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(256, 1) k_gemm_tf32x3(FactorArgs a, const TileItem* __restrict__ items) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* pipe = reinterpret_cast<float*>(smem_raw);
  float* Cs = reinterpret_cast<float*>(smem_raw);
  int* ints = reinterpret_cast<int*>(smem_raw + kTMainBytes);
  const TileItem it = items[blockIdx.x];
  const SnMeta m = a.meta[it.s];
  const float* g = static_cast<const float*>(a.L) + m.off;
  const int64_t ld = m.ld;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const int gq = lane >> 2, tq = lane & 3;

  auto load_stage = [&](int stage, int kk) {
    float* As = pipe + (size_t)stage * 2 * kTK * kTLds;
    float* Bs = As + kTK * kTLds;
#pragma unroll 4
    for (int q = 0; q < 16; ++q) {
      int e = tid + q * 256;  // 0 .. 4095: (column, row) of a 32 x 128 operand slab
      int col = e >> 7, r = e & 127;
      int k = kk + col;
      bool kok = k < it.kn;
      int64_t coff = (int64_t)(it.k0 + (kok ? k : 0)) * ld;
      bool aok = kok && r < it.mrows;
      bool bok = kok && r < it.ncols;
      cp_async4(As + col * kTLds + r, aok ? g + it.a_row0 + r + coff : g, aok ? 4 : 0);
      cp_async4(Bs + col * kTLds + r, bok ? g + it.b_row0 + r + coff : g, bok ? 4 : 0);
    }
  };

  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;

  const int nk = (it.kn + kTK - 1) / kTK;
#pragma unroll
  for (int st = 0; st < kTStages - 1; ++st) {
    if (st < nk) load_stage(st, st * kTK);
    cp_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_wait<kTStages - 2>();
    __syncthreads();
    const int nxt = kt + kTStages - 1;
    if (nxt < nk) load_stage(nxt % kTStages, nxt * kTK);
    cp_commit();
    const float* As = pipe + (size_t)(kt % kTStages) * 2 * kTK * kTLds;
    const float* Bs = As + kTK * kTLds;
#pragma unroll
    for (int ks = 0; ks < kTK; ks += 8) {
      uint32_t ahi[4][4], alo[4][4], bhi[4][2], blo[4][2];
      const float* A0 = As + (ks + tq) * kTLds + wm * 64 + gq;
      const float* A4 = A0 + 4 * kTLds;
      const float* B0 = Bs + (ks + tq) * kTLds + wn * 32 + gq;
      const float* B4 = B0 + 4 * kTLds;
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) {
        split_tf32(A0[mi * 16], ahi[mi][0], alo[mi][0]);
        split_tf32(A0[mi * 16 + 8], ahi[mi][1], alo[mi][1]);
        split_tf32(A4[mi * 16], ahi[mi][2], alo[mi][2]);
        split_tf32(A4[mi * 16 + 8], ahi[mi][3], alo[mi][3]);
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        split_tf32(B0[ni * 8], bhi[ni][0], blo[ni][0]);
        split_tf32(B4[ni * 8], bhi[ni][1], blo[ni][1]);
      }
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          mma_tf32(acc[mi][ni], alo[mi], bhi[ni]);
          mma_tf32(acc[mi][ni], ahi[mi], blo[ni]);
          mma_tf32(acc[mi][ni], ahi[mi], bhi[ni]);
        }
    }
  }
  cp_wait<0>();
  __syncthreads();
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
      int r0 = wm * 64 + mi * 16 + gq, c0 = wn * 32 + ni * 8 + 2 * tq;
      Cs[r0 + c0 * kTLdc] = acc[mi][ni][0];
      Cs[r0 + (c0 + 1) * kTLdc] = acc[mi][ni][1];
      Cs[r0 + 8 + c0 * kTLdc] = acc[mi][ni][2];
      Cs[r0 + 8 + (c0 + 1) * kTLdc] = acc[mi][ni][3];
    }
  __syncthreads();
  tile_epilogue<128, 128, 256, float, float>(a, it, m, Cs, kTLdc, (int64_t*)ints, (int64_t*)ints + 128);
}

// ---- 128 x 128 split-precision 3xTF32 tile on the 5th-generation tensor core -------
// tcgen05.mma (kind::tf32, cta_group::1, M = 128, N = 128, K = 8) with the FP32
// accumulator in tensor memory.  Operands are staged by all 256 threads: FP32
// panel values are read from HBM (coalesced along the panel's rows), split into
// tf32 hi / lo parts and written in the canonical K-major 128-byte-swizzled
// layout (one 128 B line holds the 32 columns of a chunk for one row, 8 rows
// form a 1 KB swizzle atom, 16 B pieces XOR-ed with the row), one 16 B store
// per 4 columns.  One elected thread issues the 12 MMAs of a 32-column chunk
// (4 K steps x {lo*hi, hi*lo, hi*hi}) and commits them to the chunk's
// mbarrier; the next chunk is staged into the other buffer meanwhile.  The
// epilogue reads the accumulator with tcgen05.ld (warp w: lanes 32(w%4).., column
// half w/4), stages it in shared memory and scatters it like the other tiles.
constexpr int kUM = 128, kUN = 128, kUK = 32;
constexpr int kUOpBytes = kUM * kUK * 4;           // one operand part: 16 KB
constexpr int kUStageBytes = 4 * kUOpBytes;        // A hi, A lo, B hi, B lo
constexpr int kUStages = 2;                         // split operand buffers (MMA double buffer)
constexpr int kURaw = 2;                            // raw FP32 chunks in flight (cp.async)
constexpr int kURawLd = kUM + 4;                    // raw column: 128 rows from a 4-row boundary
constexpr int kURawBytes = 2 * kUK * kURawLd * 4;   // A and B columns of one chunk: 33 KB
constexpr int kULdc = 132;
constexpr size_t kUCBytes = (size_t)kUN * kULdc * sizeof(float);
constexpr size_t kUOpAll = (size_t)kUStages * kUStageBytes;   // 128 KB; C staging reuses it
constexpr size_t kUMainBytes = kUOpAll + (size_t)kURaw * kURawBytes;
constexpr size_t kUSmemBytes = 1024 + kUMainBytes + 64;
static_assert(kUCBytes <= kUOpAll, "C staging must fit in the operand buffers");
static_assert(kUSmemBytes <= 232448, "shared memory of the tcgen05 tile");
constexpr int kUTmemCols = 128;
constexpr long long kUWaitLimit = 1LL << 24;  // mbarrier polls before a tile gives up (seconds)

// Byte offset of the 16 B piece holding columns 4*kg .. 4*kg+3 of row m in a
// 128 x 32 operand part (K-major, 128-byte swizzle).
__device__ __forceinline__ uint32_t umma_k_offset(int m, int kg) {
  return (uint32_t)((m >> 3) * 1024 + (m & 7) * 128 + ((kg ^ (m & 7)) << 4));
}

// Shared-memory matrix descriptor of a K-major 128-byte-swizzled operand:
// start >> 4, leading byte offset 16 (unused by this layout), stride byte
// offset 1024 (8-row atoms), descriptor version 1, 128-byte swizzle.  A K step
// of 8 tf32 columns inside the 128 B line advances the start by 32 bytes.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(16 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}

// Instruction descriptor: D f32, A and B tf32, both K-major, N = 128, M = 128.
constexpr uint32_t kUIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kUN >> 3) << 17) |
                             ((uint32_t)(kUM >> 4) << 24);


__global__ void __launch_bounds__(256, 1) k_gemm_tc32(FactorArgs a, const TileItem* __restrict__ items) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t raw_addr = (uint32_t)__cvta_generic_to_shared(smem_raw);
  const uint32_t pad = ((raw_addr + 1023u) & ~1023u) - raw_addr;  // swizzle atoms need 1 KB alignment
  unsigned char* base = smem_raw + pad;
  const uint32_t base_addr = raw_addr + pad;
  float* Cs = reinterpret_cast<float*>(base);  // reused once every MMA has completed
  float* raw = reinterpret_cast<float*>(base + kUOpAll);  // kURaw x {A, B} x [32 columns][128 rows]
  int* ints = reinterpret_cast<int*>(raw);                  // epilogue maps reuse the raw stages
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kUMainBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + kUStages);
  __shared__ int sh_abort;

  const TileItem it = items[blockIdx.x];
  const SnMeta m = a.meta[it.s];
  const float* g = static_cast<const float*>(a.L) + m.off;
  const int64_t ld = m.ld;
  const int tid = threadIdx.x, warp = tid >> 5;

  if (tid == 0) {
    sh_abort = 0;
    for (int i = 0; i < kUStages; ++i) {
      const uint32_t b = (uint32_t)__cvta_generic_to_shared(bars + i);
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(b) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(slot),
                 "r"(kUTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // raw chunk kk of A and B in 16-byte copies: column k of the chunk holds panel rows
  // from the 4-row boundary at or below the tile's first row, so tile row r sits at
  // raw[stage][op][k][r + shift].  Panels start on 32-element boundaries and their
  // leading dimension is a multiple of 4, so every copy is aligned; a copy is issued
  // only if it holds a row of the tile, which keeps it inside the panel's padded column.
  const int a0 = it.a_row0 & ~3, b0 = it.b_row0 & ~3;
  const int ashift = it.a_row0 - a0, bshift = it.b_row0 - b0;
  auto load_raw = [&](int stage, int kk) {
    float* ra = raw + (size_t)stage * (kURawBytes / 4);
    float* rb = ra + kUK * kURawLd;
    constexpr int kVec = kUK * (kURawLd / 4);  // 16-byte copies per operand
#pragma unroll
    for (int q = 0; q < (kVec + 255) / 256; ++q) {
      const int e = tid + q * 256;
      if (e >= kVec) break;
      const int col = e / (kURawLd / 4), f = e - col * (kURawLd / 4), k = kk + col;
      const bool kok = k < it.kn;
      const int64_t coff = (int64_t)(it.k0 + (kok ? k : 0)) * ld;
      const bool aok = kok && a0 + 4 * f < it.a_row0 + it.mrows;
      const bool bok = kok && b0 + 4 * f < it.b_row0 + it.ncols;
      cp_async16(ra + col * kURawLd + 4 * f, aok ? g + a0 + 4 * f + coff : g, aok ? 16 : 0);
      cp_async16(rb + col * kURawLd + 4 * f, bok ? g + b0 + 4 * f + coff : g, bok ? 16 : 0);
    }
  };
  // this thread's split pieces: row r, column groups kq + 2q (q = 0..3) of 4 columns
  const int r = tid & 127, kq = tid >> 7;
  const int nk = (it.kn + kUK - 1) / kUK;
#pragma unroll
  for (int c = 0; c < kURaw - 1; ++c) {
    if (c < nk) load_raw(c, c * kUK);
    cp_commit();
  }
  int committed = -1;  // last chunk whose MMAs were committed
  for (int kt = 0; kt < nk; ++kt) {
    const int nxt = kt + kURaw - 1;  // its raw stage was split at kt - 1, before that iteration's barrier
    if (nxt < nk) load_raw(nxt % kURaw, nxt * kUK);
    cp_commit();
    cp_wait<kURaw - 1>();
    const int st = kt & 1;
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(bars + st);
    if (kt >= 2 && !mbar_wait(bar, (uint32_t)(((kt >> 1) - 1) & 1), kUWaitLimit)) sh_abort = 1;
    __syncthreads();  // every thread's raw copies of chunk kt have landed
    const float* ra = raw + (size_t)(kt % kURaw) * (kURawBytes / 4) + r + ashift;
    const float* rb = raw + (size_t)(kt % kURaw) * (kURawBytes / 4) + kUK * kURawLd + r + bshift;
    const bool arow = r < it.mrows, brow = r < it.ncols;  // rows past the tile hold other panel rows
    unsigned char* sb = base + st * kUStageBytes;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k4 = 4 * (kq + 2 * q);
      const uint32_t off = umma_k_offset(r, kq + 2 * q);
      uint4 ah, al, bh, bl;
      split_tf32(arow ? ra[(k4 + 0) * kURawLd] : 0.f, ah.x, al.x);
      split_tf32(arow ? ra[(k4 + 1) * kURawLd] : 0.f, ah.y, al.y);
      split_tf32(arow ? ra[(k4 + 2) * kURawLd] : 0.f, ah.z, al.z);
      split_tf32(arow ? ra[(k4 + 3) * kURawLd] : 0.f, ah.w, al.w);
      split_tf32(brow ? rb[(k4 + 0) * kURawLd] : 0.f, bh.x, bl.x);
      split_tf32(brow ? rb[(k4 + 1) * kURawLd] : 0.f, bh.y, bl.y);
      split_tf32(brow ? rb[(k4 + 2) * kURawLd] : 0.f, bh.z, bl.z);
      split_tf32(brow ? rb[(k4 + 3) * kURawLd] : 0.f, bh.w, bl.w);
      *reinterpret_cast<uint4*>(sb + off) = ah;
      *reinterpret_cast<uint4*>(sb + kUOpBytes + off) = al;
      *reinterpret_cast<uint4*>(sb + 2 * kUOpBytes + off) = bh;
      *reinterpret_cast<uint4*>(sb + 3 * kUOpBytes + off) = bl;
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (sh_abort) break;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t sa = base_addr + st * kUStageBytes;
#pragma unroll
      for (int ks = 0; ks < kUK / 8; ++ks) {
        const uint64_t ahi = umma_desc(sa + ks * 32), alo = umma_desc(sa + kUOpBytes + ks * 32);
        const uint64_t bhi = umma_desc(sa + 2 * kUOpBytes + ks * 32), blo = umma_desc(sa + 3 * kUOpBytes + ks * 32);
        const uint64_t pa[3] = {alo, ahi, ahi}, pb[3] = {bhi, blo, bhi};
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const uint32_t acc = (kt > 0 || ks > 0 || p > 0) ? 1u : 0u;
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
              " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
              "l"(pa[p]), "l"(pb[p]), "r"(kUIdesc), "r"(acc)
              : "memory");
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                   : "memory");
    }
    committed = kt;
  }
  cp_wait<0>();
  bool ok = !sh_abort;
  if (committed >= 0) {  // every MMA done before the accumulator is read or the stages reused
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(bars + (committed & 1));
    if (!mbar_wait(bar, (uint32_t)((committed >> 1) & 1), kUWaitLimit)) ok = false;
  }
  ok = __syncthreads_and(ok) != 0;  // one decision for the whole CTA (tcgen05.ld is warp-collective)
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  int64_t* cbase = reinterpret_cast<int64_t*>(ints);  // mode 1 column maps (reuse the raw stages)
  int64_t* crel = cbase + 128;
  if (ok) {
    const int quarter = warp & 3, half = warp >> 2;
    const int row = quarter * 32 + (tid & 31);
    if (it.mode == 1) {
      // external update straight from tensor memory: thread = accumulator row, 64 columns
      if (tid < it.ncols) {
        const int jc = it.b_row0 + tid;
        const RelGroup gr = a.groups[a.row_group[m.lidx + jc]];
        const SnMeta mt = a.meta[gr.t];
        cbase[tid] = mt.off + (int64_t)(a.rows[m.lidx + jc] - mt.fc) * mt.ld;
        crel[tid] = gr.rel_off - gr.j0;
      }
      __syncthreads();
    }
    float* L = static_cast<float*>(a.L);
    const int jr = it.a_row0 + row;
    int64_t last = INT64_MIN;
    int pos = 0;
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      const int c0 = half * 64 + part * 32;
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
            "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
            "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (it.mode == 1) {
        if (row < it.mrows) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int c = c0 + j;
            if (c < it.ncols && jr >= it.b_row0 + c) {
              const int64_t cr = crel[c];
              if (cr != last) {
                pos = a.rel[cr + jr];
                last = cr;
              }
              atomicAdd(L + cbase[c] + pos, -__uint_as_float(v[j]));
            }
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) Cs[row + (c0 + j) * kULdc] = __uint_as_float(v[j]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kUTmemCols) : "memory");
  }
  if (!ok) {
    if (tid == 0) report_status(a.status, 3, it.s, -1);
    return;
  }
  if (it.mode == 0) tile_epilogue<kUM, kUN, 256, float, float>(a, it, m, Cs, kULdc, cbase, crel);
}

// ---- 128 x 128 3xTF32 tile with TMA-fed operands -------------------------------------
// The FP32 panels of supernodes with these tiles have a split copy: once a row of a
// panel is final (TRSM tile, or small panel), its tf32 hi part (cvt.rna) and lo part
// (the rounded remainder) are written row-major, hi block then lo block (row pitch
// round_up(w, 4)).  A 3-D tiled tensor map per panel (columns inner, rows, hi / lo; 128-byte
// swizzle, zero outside the panel) lets one TMA load bring a 128-row x 32-column chunk of
// both parts straight into the K-major 128-byte-swizzled layout the MMAs read (8-row atoms
// of 1 KB; hi at +0, lo at +16 KB), so a tile is TMA -> tcgen05 -> TMEM with no thread
// touching its operands.  Thread 0 issues the loads and the chunk's 12 MMAs (4 K steps x
// {lo*hi, hi*lo, hi*hi}, the order of k_gemm_tc32) and commits them to the stage's mbarrier;
// it refills a stage once the MMAs that read it are done.  Three stages of 64 KB (A hi,
// A lo, B hi, B lo); a tile whose two operands are the same rows loads one.  Accumulator row
// i is panel row a_row0 + i and column j panel row b_row0 + j.
constexpr int kVStages = 3;
constexpr int kVOpBytes = 128 * 32 * 4;              // one operand part: 16 KB
constexpr int kVStageBytes = 4 * kVOpBytes;          // A hi, A lo, B hi, B lo
constexpr size_t kVMainBytes = (size_t)kVStages * kVStageBytes;
constexpr size_t kVSmemBytes = 1024 + kVMainBytes + 2 * kVStages * sizeof(uint64_t) + 16;
static_assert(kUCBytes + 2 * 128 * sizeof(int64_t) <= kVMainBytes, "C staging and column maps fit the stages");
static_assert(kVSmemBytes <= 232448, "shared memory of the TMA-fed tcgen05 tile");

// 32 columns x 128 rows x {hi, lo} of a panel's split copy (tensor map, coordinates
// column, row, part) into dst, completing on bar.
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const void* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(0), "r"(bar)
      : "memory");
}

// Per-CTA state of the TMA-fed tile: stage buffers (1 KB aligned), the per-stage
// mbarriers and the tensor-memory accumulator, kept across the tiles a persistent CTA
// runs; g counts the chunks this CTA has run, so chunk q of its life uses stage q % 3
// and waits for phase (q / 3) & 1 of that stage's barriers.
struct TcTile {
  unsigned char* base;
  uint32_t base_addr;
  uint64_t* full;  // chunk landed (TMA transaction bytes)
  uint64_t* done;  // chunk's MMAs finished (tcgen05.commit)
  uint32_t tmem;
  uint32_t g;
};

// All threads: barriers, 128 tensor-memory columns (kVSmemBytes of dynamic shared memory).
__device__ __forceinline__ void tc_setup(TcTile& S, unsigned char* smem_raw) {
  const uint32_t raw_addr = (uint32_t)__cvta_generic_to_shared(smem_raw);
  const uint32_t pad = ((raw_addr + 1023u) & ~1023u) - raw_addr;  // swizzle atoms need 1 KB alignment
  S.base = smem_raw + pad;
  S.base_addr = raw_addr + pad;
  S.full = reinterpret_cast<uint64_t*>(S.base + kVMainBytes);
  S.done = S.full + kVStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(S.done + kVStages);
  S.g = 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2 * kVStages; ++i) {
      const uint32_t b = (uint32_t)__cvta_generic_to_shared(S.full + i);
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(b) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if ((threadIdx.x >> 5) == 0) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(slot),
                 "r"(kUTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  S.tmem = *tmem_slot;
}

__device__ __forceinline__ void tc_teardown(const TcTile& S) {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(S.tmem), "r"(kUTmemCols)
                 : "memory");
  }
}

// One TMA-fed tile (all 256 threads).  Returns false, after recording status 3, when a
// barrier wait gave up; the CTA's copies and MMAs in flight have then been waited for
// (bounded).  The stages' shared memory may hold anything written by earlier work.
__device__ bool tc32t_tile_task(const FactorArgs& a, const TileItem& it, TcTile& S) {
  __shared__ int sh_abort, sh_last;
  unsigned char* base = S.base;
  const uint32_t base_addr = S.base_addr;
  float* Cs = reinterpret_cast<float*>(base);  // mode 0 staging, once every MMA has completed
  int64_t* cbase = reinterpret_cast<int64_t*>(base + kUCBytes);
  int64_t* crel = cbase + 128;
  const SnMeta m = a.meta[it.s];
  const void* map = static_cast<const unsigned char*>(a.tmaps) + 128 * (size_t)a.tmap_of[it.s];
  const int tid = threadIdx.x, warp = tid >> 5;
  const bool same = it.a_row0 == it.b_row0;  // both operands are the same panel rows
  const int nops = same ? 1 : 2;
  const int nk = (it.kn + 31) / 32;
  const uint32_t g0 = S.g;

  // earlier generic-proxy accesses of the stages come before this tile's TMA writes
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (tid == 0) sh_abort = 0;
  __syncthreads();

  if (tid == 0) {
    // the split copy was written by other CTAs (generic proxy) before the counters
    // this task waited for were released
    asm volatile("fence.proxy.async.global;\n" ::: "memory");
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(map) : "memory");
    // chunk kt into stage (g0 + kt) % kVStages: one box of 32 columns x 128 rows x {hi, lo} per operand
    auto issue = [&](int kt) {
      const int st = (g0 + kt) % kVStages;
      const uint32_t sa = base_addr + st * kVStageBytes;
      const uint32_t bar = (uint32_t)__cvta_generic_to_shared(S.full + st);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(nops * 2 * kVOpBytes)
                   : "memory");
      const int x = it.k0 + kt * 32;
      tma_load_3d(sa, map, x, it.a_row0, bar);
      if (!same) tma_load_3d(sa + 2 * kVOpBytes, map, x, it.b_row0, bar);
    };
    int issued = 0;
    for (; issued < nk && issued < kVStages; ++issued) issue(issued);
    int committed = -1;
    for (int kt = 0; kt < nk; ++kt) {
      const uint32_t q = g0 + kt;
      const int st = q % kVStages;
      if (!mbar_wait((uint32_t)__cvta_generic_to_shared(S.full + st), (q / kVStages) & 1, kUWaitLimit)) {
        sh_abort = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t sa = base_addr + st * kVStageBytes;
      const uint32_t sbb = same ? sa : sa + 2 * kVOpBytes;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {  // K step of 8 columns = 32 bytes of each 128-byte line
        const uint64_t ahi = umma_desc(sa + ks * 32), alo = umma_desc(sa + kVOpBytes + ks * 32);
        const uint64_t bhi = umma_desc(sbb + ks * 32), blo = umma_desc(sbb + kVOpBytes + ks * 32);
        const uint64_t pa[3] = {alo, ahi, ahi}, pb[3] = {bhi, blo, bhi};
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const uint32_t acc = (kt > 0 || ks > 0 || p > 0) ? 1u : 0u;
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
              " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(S.tmem),
              "l"(pa[p]), "l"(pb[p]), "r"(kUIdesc), "r"(acc)
              : "memory");
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       (uint32_t)__cvta_generic_to_shared(S.done + st))
                   : "memory");
      committed = kt;
      // refill the stage of the previous chunk once its MMAs are done (this chunk's queue behind them)
      const int pk = kt - 1;
      if (pk >= 0 && issued < nk) {
        const uint32_t pq = g0 + pk;
        if (!mbar_wait((uint32_t)__cvta_generic_to_shared(S.done + pq % kVStages), (pq / kVStages) & 1,
                       kUWaitLimit)) {
          sh_abort = 1;
          break;
        }
        issue(issued++);
      }
    }
    if (sh_abort) {  // let this CTA's copies in flight land before the stages are reused (bounded)
      for (int kt = committed + 1; kt < issued; ++kt) {
        const uint32_t q = g0 + kt;
        mbar_wait((uint32_t)__cvta_generic_to_shared(S.full + q % kVStages), (q / kVStages) & 1, kUWaitLimit);
      }
    }
    sh_last = committed;
  }
  __syncthreads();
  const int committed = sh_last;
  bool ok = !sh_abort;
  if (committed >= 0) {  // every thread: the last commit covers every earlier MMA
    const uint32_t q = g0 + committed;
    if (!mbar_wait((uint32_t)__cvta_generic_to_shared(S.done + q % kVStages), (q / kVStages) & 1, kUWaitLimit))
      ok = false;
  }
  S.g = g0 + nk;  // every chunk's barrier phases were consumed (the loop ran to nk unless aborted)
  ok = __syncthreads_and(ok) != 0;  // one decision for the whole CTA (tcgen05.ld is warp-collective)
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (ok) {
    const int quarter = warp & 3, half = warp >> 2;
    const int row = quarter * 32 + (tid & 31);
    if (it.mode == 1) {
      if (tid < it.ncols) {
        const int jc = it.b_row0 + tid;
        const RelGroup gr = a.groups[a.row_group[m.lidx + jc]];
        const SnMeta mt = a.meta[gr.t];
        cbase[tid] = mt.off + (int64_t)(a.rows[m.lidx + jc] - mt.fc) * mt.ld;
        crel[tid] = gr.rel_off - gr.j0;
      }
      __syncthreads();
    }
    float* L = static_cast<float*>(a.L);
    const int jr = it.a_row0 + row;
    int64_t last = INT64_MIN;
    int pos = 0;
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      const int c0 = half * 64 + part * 32;
      uint32_t v[32];
      const uint32_t taddr = S.tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
            "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
            "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (it.mode == 1) {
        if (row < it.mrows) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int c = c0 + j;
            if (c < it.ncols && jr >= it.b_row0 + c) {
              const int64_t cr = crel[c];
              if (cr != last) {
                pos = a.rel[cr + jr];
                last = cr;
              }
              atomicAdd(L + cbase[c] + pos, -__uint_as_float(v[j]));
            }
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) Cs[row + (c0 + j) * kULdc] = __uint_as_float(v[j]);
      }
    }
  }
  // the accumulator has been read before the next tile's MMAs overwrite it
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (!ok) {
    if (tid == 0) report_status(a.status, 3, it.s, -1);
    return false;
  }
  if (it.mode == 0) tile_epilogue<kUM, kUN, 256, float, float>(a, it, m, Cs, kULdc, cbase, crel);
  return true;
}

__device__ __forceinline__ void named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// ---- persistent, warp-specialised TMA-fed tcgen05 tile ----------------------------------
// One CTA per SM loops over the launch's tiles (tile blockIdx.x + i * gridDim.x).  Warp 0
// (one lane) issues the TMA loads of every chunk into a ring of three 64 KB stages, warp 1
// (one lane) the MMAs into one of two tensor-memory accumulators (256 columns), and warps
// 2-5 read an accumulator out and subtract it while the next tile is loaded and multiplied.
// mbarriers: per stage "full" (TMA bytes landed) and "done" (its MMAs finished), per
// accumulator "ready" (last MMA of a tile done) and "free" (its 4 epilogue warps have read
// it).  The in-panel tiles go through a 32-column staging buffer so that each thread
// subtracts 4 consecutive rows at a time (16-byte reductions); external updates are
// scattered straight from the registers.
constexpr int kWThreads = 192;
constexpr int kWCsLd = 132;                                          // staging: 32 columns x 128 rows
constexpr size_t kWCsBytes = (size_t)32 * kWCsLd * sizeof(float);    // 16.5 KB
constexpr size_t kWMapBytes = 2 * 256 * sizeof(int64_t);             // per accumulator {base, rel}
constexpr size_t kWSmemBytes = 1024 + kVMainBytes + kWCsBytes + kWMapBytes + 16 * sizeof(uint64_t) + 16;
static_assert(kWSmemBytes <= 232448, "shared memory of the warp-specialised tcgen05 tile");

__global__ void __launch_bounds__(kWThreads, 1) k_gemm_tc32w(FactorArgs a, const TileItem* __restrict__ items,
                                                             int count) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t raw_addr = (uint32_t)__cvta_generic_to_shared(smem_raw);
  const uint32_t pad = ((raw_addr + 1023u) & ~1023u) - raw_addr;  // swizzle atoms need 1 KB alignment
  unsigned char* base = smem_raw + pad;
  const uint32_t base_addr = raw_addr + pad;
  float* Cs = reinterpret_cast<float*>(base + kVMainBytes);
  int64_t* maps = reinterpret_cast<int64_t*>(base + kVMainBytes + kWCsBytes);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kVMainBytes + kWCsBytes + kWMapBytes);
  uint64_t* full = bars;           // [kVStages]
  uint64_t* done = bars + 3;       // [kVStages]
  uint64_t* ready = bars + 6;      // [2]
  uint64_t* freed = bars + 8;      // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 10);
  __shared__ int sh_abort, sh_eab;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto sa = [](const void* p) { return (uint32_t)__cvta_generic_to_shared(p); };
  static_assert(kVStages == 3, "barrier layout");

  if (tid == 0) {
    sh_abort = 0;
    sh_eab = 0;
    for (int i = 0; i < 3; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(sa(full + i)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(sa(done + i)) : "memory");
    }
    for (int i = 0; i < 2; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(sa(ready + i)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;\n" ::"r"(sa(freed + i)) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sa(tmem_slot)),
                 "r"(2 * kUTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ---- TMA producer ----
    if (lane == 0) {
      uint32_t G = 0;  // chunks issued by this CTA
      for (int tile = blockIdx.x; tile < count && !sh_abort; tile += gridDim.x) {
        const TileItem it = items[tile];
        const void* map = static_cast<const unsigned char*>(a.tmaps) + 128 * (size_t)a.tmap_of[it.s];
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(map) : "memory");
        const bool same = it.a_row0 == it.b_row0;
        const int nk = (it.kn + 31) / 32;
        for (int kt = 0; kt < nk; ++kt, ++G) {
          const int st = G % kVStages;
          if (G >= kVStages &&
              !mbar_wait(sa(done + st), (G / kVStages - 1) & 1, kUWaitLimit)) {  // the stage's MMAs finished
            sh_abort = 1;
            break;
          }
          const uint32_t s0 = base_addr + st * kVStageBytes;
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(sa(full + st)),
                       "r"((same ? 1 : 2) * 2 * kVOpBytes)
                       : "memory");
          tma_load_3d(s0, map, it.k0 + kt * 32, it.a_row0, sa(full + st));
          if (!same) tma_load_3d(s0 + 2 * kVOpBytes, map, it.k0 + kt * 32, it.b_row0, sa(full + st));
        }
      }
      // the last stages' copies have landed before the CTA leaves (bounded)
      for (uint32_t q = G > kVStages ? G - kVStages : 0; q < G; ++q)
        mbar_wait(sa(full + q % kVStages), (q / kVStages) & 1, kUWaitLimit);
    }
  } else if (warp == 1) {
    // ---- MMA issuer ----
    if (lane == 0) {
      uint32_t G = 0;
      int last = -1;  // stage of the last committed chunk, and its phase
      uint32_t lastq = 0;
      int ti = 0;
      for (int tile = blockIdx.x; tile < count && !sh_abort; tile += gridDim.x, ++ti) {
        const TileItem it = items[tile];
        const bool same = it.a_row0 == it.b_row0;
        const int nk = (it.kn + 31) / 32, acc = ti & 1;
        if (ti >= 2 && !mbar_wait(sa(freed + acc), ((ti >> 1) - 1) & 1, kUWaitLimit)) {
          sh_abort = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t dcol = tmem + (uint32_t)(acc * kUTmemCols);
        for (int kt = 0; kt < nk; ++kt, ++G) {
          const int st = G % kVStages;
          if (!mbar_wait(sa(full + st), (G / kVStages) & 1, kUWaitLimit)) {
            sh_abort = 1;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t s0 = base_addr + st * kVStageBytes;
          const uint32_t sb = same ? s0 : s0 + 2 * kVOpBytes;
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            const uint64_t ahi = umma_desc(s0 + ks * 32), alo = umma_desc(s0 + kVOpBytes + ks * 32);
            const uint64_t bhi = umma_desc(sb + ks * 32), blo = umma_desc(sb + kVOpBytes + ks * 32);
            const uint64_t pa[3] = {alo, ahi, ahi}, pb[3] = {bhi, blo, bhi};
#pragma unroll
            for (int p = 0; p < 3; ++p) {
              const uint32_t accum = (kt > 0 || ks > 0 || p > 0) ? 1u : 0u;
              asm volatile(
                  "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                  " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(dcol),
                  "l"(pa[p]), "l"(pb[p]), "r"(kUIdesc), "r"(accum)
                  : "memory");
            }
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                           sa(done + st))
                       : "memory");
          last = st;
          lastq = G;
        }
        if (sh_abort) break;
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         sa(ready + acc))
                     : "memory");
      }
      if (last >= 0)  // every MMA finished before the stages and the tensor memory go away (bounded)
        mbar_wait(sa(done + last), (lastq / kVStages) & 1, kUWaitLimit);
    }
  } else {
    // ---- epilogue: warps 2-5, one accumulator row per thread ----
    const int et = tid - 64, quarter = warp & 3, row = quarter * 32 + lane;
    float* L = static_cast<float*>(a.L);
    int ti = 0;
    for (int tile = blockIdx.x; tile < count; tile += gridDim.x, ++ti) {
      const TileItem it = items[tile];
      const SnMeta m = a.meta[it.s];
      const int acc = ti & 1;
      int64_t* cbase = maps + acc * 256;
      int64_t* crel = cbase + 128;
      if (it.mode == 1 && et < it.ncols) {
        const int jc = it.b_row0 + et;
        const RelGroup gr = a.groups[a.row_group[m.lidx + jc]];
        const SnMeta mt = a.meta[gr.t];
        cbase[et] = mt.off + (int64_t)(a.rows[m.lidx + jc] - mt.fc) * mt.ld;
        crel[et] = gr.rel_off - gr.j0;
      }
      const bool ok = mbar_wait(sa(ready + acc), (ti >> 1) & 1, kUWaitLimit);
      if (!ok) sh_eab = 1;  // written by epilogue threads only, so all of them read the same value
      named_sync(1, 128);   // maps ready; every epilogue thread has seen the accumulator ready (or not)
      if (sh_eab) {
        if (et == 0) sh_abort = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const int jr = it.a_row0 + row;
      int64_t last = INT64_MIN;
      int pos = 0;
      for (int c0 = 0; c0 < kUN; c0 += 32) {
        uint32_t v[32];
        const uint32_t taddr = tmem + (uint32_t)(acc * kUTmemCols) + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
              "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
              "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
              "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (it.mode == 1) {
          if (row < it.mrows) {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              const int c = c0 + j;
              if (c < it.ncols && jr >= it.b_row0 + c) {
                const int64_t cr = crel[c];
                if (cr != last) {
                  pos = a.rel[cr + jr];
                  last = cr;
                }
                atomicAdd(L + cbase[c] + pos, -__uint_as_float(v[j]));
              }
            }
          }
        } else {
          // in-panel: stage 32 columns, then 4 consecutive rows per reduction (the panel starts
          // on 32 elements, ld is a multiple of 4 and in-panel tiles start on 64-row boundaries)
#pragma unroll
          for (int j = 0; j < 32; ++j) Cs[row + j * kWCsLd] = __uint_as_float(v[j]);
          named_sync(1, 128);
          float* g = L + m.off + it.a_row0;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int idx = et + q * 128, q4 = idx & 31, j = idx >> 5, i0 = 4 * q4, c = c0 + j;
            if (c >= it.ncols) continue;
            const int gc = it.b_row0 + c, jr0 = it.a_row0 + i0;
            const float4 val = *reinterpret_cast<const float4*>(Cs + i0 + j * kWCsLd);
            float* dst = g + i0 + (int64_t)gc * m.ld;
            if (i0 + 3 < it.mrows && jr0 >= gc) {
              atomicAdd(reinterpret_cast<float4*>(dst), make_float4(-val.x, -val.y, -val.z, -val.w));
            } else {
              const float vv[4] = {val.x, val.y, val.z, val.w};
#pragma unroll
              for (int e = 0; e < 4; ++e)
                if (i0 + e < it.mrows && jr0 + e >= gc) atomicAdd(dst + e, -vv[e]);
            }
          }
          named_sync(1, 128);  // the staging buffer is free for the next 32 columns
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(sa(freed + acc)) : "memory");
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (sh_abort && tid == 0) report_status(a.status, 3, -1, -1);
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(2 * kUTmemCols)
                 : "memory");
  }
}

// ---- persistent, warp-specialised variant of the tcgen05 tile ---------------------
// One CTA per SM loops over the launch's tiles.  Warps 0-7 stage operands and (one
// thread) issue the MMAs exactly as k_gemm_tc32 does; warps 8-11 are the epilogue:
// each thread owns one accumulator row, reads it from tensor memory 32 columns at a
// time and scatters it.  Two accumulators (256 TMEM columns) let the epilogue of
// tile i run while tile i + 1 is staged and multiplied.  mbarriers: per operand
// stage (MMAs done, stage reusable), per accumulator "full" (last MMA of a tile
// done) and "empty" (its 4 epilogue warps have read it).
constexpr int kPStages = 2, kPRaw = 2, kPThreads = 384;
constexpr long long kPWaitLimit = 1LL << 22;  // mbarrier polls before a wait gives up
constexpr size_t kPOpAll = (size_t)kPStages * kUStageBytes;          // 128 KB
constexpr size_t kPRawAll = (size_t)kPRaw * kURawBytes;              // 64 KB
constexpr size_t kPMaps = 4 * 128 * sizeof(int64_t);                 // 2 accumulators x {base, rel}
constexpr size_t kPSmemBytes = 1024 + kPOpAll + kPRawAll + kPMaps + 128;
static_assert(kPSmemBytes <= 232448, "shared memory of the persistent tcgen05 tile");

__global__ void __launch_bounds__(kPThreads, 1) k_gemm_tc32p(FactorArgs a, const TileItem* __restrict__ items,
                                                           int count) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t raw_addr = (uint32_t)__cvta_generic_to_shared(smem_raw);
  const uint32_t pad = ((raw_addr + 1023u) & ~1023u) - raw_addr;  // swizzle atoms need 1 KB alignment
  unsigned char* base = smem_raw + pad;
  const uint32_t base_addr = raw_addr + pad;
  float* raw = reinterpret_cast<float*>(base + kPOpAll);
  int64_t* maps = reinterpret_cast<int64_t*>(base + kPOpAll + kPRawAll);  // [acc][base 128 | rel 128]
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kPOpAll + kPRawAll + kPMaps);
  uint64_t* stage_bar = bars;      // [kPStages]
  uint64_t* full_bar = bars + 2;   // [2]
  uint64_t* empty_bar = bars + 4;  // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 6);
  __shared__ int sh_pab, sh_eok[2];  // producer abort (read after producer barriers); epilogue wait results
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto sa_of = [](const void* p) { return (uint32_t)__cvta_generic_to_shared(p); };

  if (tid == 0) {
    sh_pab = 0;
    sh_eok[0] = sh_eok[1] = 1;
    for (int i = 0; i < 2; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(sa_of(stage_bar + i)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(sa_of(full_bar + i)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;\n" ::"r"(sa_of(empty_bar + i)) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sa_of(tmem_slot)),
                 "r"(2 * kUTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp < 8) {
    // ---- producers: stage operands, one thread issues the MMAs ----
    const int r = tid & 127, kq = tid >> 7;
    int gchunk = 0;        // chunks staged by this CTA (operand stage and phase bookkeeping)
    int last_commit = -1;  // global index of the last committed chunk
    for (int ti = 0, tile = blockIdx.x; tile < count; tile += gridDim.x, ++ti) {
      named_sync(1, 256);  // the previous tile's raw stages are consumed; abort flag settled
      if (sh_pab) break;
      const TileItem it = items[tile];
      const SnMeta m = a.meta[it.s];
      const float* g = static_cast<const float*>(a.L) + m.off;
      const int64_t ld = m.ld;
      const int acc = ti & 1;
      auto load_raw = [&](int stage, int kk) {
        float* ra = raw + (size_t)stage * (kURawBytes / 4);
        float* rb = ra + kUK * kUM;
#pragma unroll 4
        for (int q = 0; q < kUK * kUM / 256; ++q) {
          const int e = tid + q * 256, col = e >> 7, rr = e & 127, k = kk + col;
          const bool kok = k < it.kn;
          const int64_t coff = (int64_t)(it.k0 + (kok ? k : 0)) * ld;
          const bool aok = kok && rr < it.mrows, bok = kok && rr < it.ncols;
          cp_async4(ra + col * kUM + rr, aok ? g + it.a_row0 + rr + coff : g, aok ? 4 : 0);
          cp_async4(rb + col * kUM + rr, bok ? g + it.b_row0 + rr + coff : g, bok ? 4 : 0);
        }
      };
      const int nk = (it.kn + kUK - 1) / kUK;
      load_raw(0, 0);
      cp_commit();
      for (int kt = 0; kt < nk; ++kt) {
        if (kt + 1 < nk) load_raw((kt + 1) % kPRaw, (kt + 1) * kUK);
        cp_commit();
        cp_wait<kPRaw - 1>();
        const int G = gchunk + kt, st = G % kPStages;
        if (G >= kPStages &&
            !mbar_wait(sa_of(stage_bar + st), (uint32_t)((G / kPStages - 1) & 1), kPWaitLimit))
          sh_pab = 1;
        named_sync(1, 256);  // raw chunk kt has landed for every producer
        const float* ra = raw + (size_t)(kt % kPRaw) * (kURawBytes / 4);
        const float* rb = ra + kUK * kUM;
        unsigned char* sb = base + st * kUStageBytes;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int k4 = 4 * (kq + 2 * q);
          const uint32_t off = umma_k_offset(r, kq + 2 * q);
          uint4 ah, al, bh, bl;
          split_tf32(ra[(k4 + 0) * kUM + r], ah.x, al.x);
          split_tf32(ra[(k4 + 1) * kUM + r], ah.y, al.y);
          split_tf32(ra[(k4 + 2) * kUM + r], ah.z, al.z);
          split_tf32(ra[(k4 + 3) * kUM + r], ah.w, al.w);
          split_tf32(rb[(k4 + 0) * kUM + r], bh.x, bl.x);
          split_tf32(rb[(k4 + 1) * kUM + r], bh.y, bl.y);
          split_tf32(rb[(k4 + 2) * kUM + r], bh.z, bl.z);
          split_tf32(rb[(k4 + 3) * kUM + r], bh.w, bl.w);
          *reinterpret_cast<uint4*>(sb + off) = ah;
          *reinterpret_cast<uint4*>(sb + kUOpBytes + off) = al;
          *reinterpret_cast<uint4*>(sb + 2 * kUOpBytes + off) = bh;
          *reinterpret_cast<uint4*>(sb + 3 * kUOpBytes + off) = bl;
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        named_sync(1, 256);
        if (sh_pab) break;
        if (tid == 0) {
          if (kt == 0 && ti >= 2 &&
              !mbar_wait(sa_of(empty_bar + acc), (uint32_t)(((ti >> 1) - 1) & 1), kPWaitLimit))
            sh_pab = 1;  // the accumulator's previous tile has not been read out
          if (!sh_pab) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t sa = base_addr + st * kUStageBytes, dcol = tmem + (uint32_t)(acc * kUTmemCols);
#pragma unroll
            for (int ks = 0; ks < kUK / 8; ++ks) {
              const uint64_t ahi = umma_desc(sa + ks * 32), alo = umma_desc(sa + kUOpBytes + ks * 32);
              const uint64_t bhi = umma_desc(sa + 2 * kUOpBytes + ks * 32),
                             blo = umma_desc(sa + 3 * kUOpBytes + ks * 32);
              const uint64_t pa[3] = {alo, ahi, ahi}, pb[3] = {bhi, blo, bhi};
#pragma unroll
              for (int p = 0; p < 3; ++p) {
                const uint32_t accum = (kt > 0 || ks > 0 || p > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(dcol),
                    "l"(pa[p]), "l"(pb[p]), "r"(kUIdesc), "r"(accum)
                    : "memory");
              }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             sa_of(stage_bar + st))
                         : "memory");
            if (kt == nk - 1)
              asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                               sa_of(full_bar + acc))
                           : "memory");
          }
        }
        if (!sh_pab) last_commit = G;
      }
      gchunk += nk;
    }
    cp_wait<0>();
    if (tid == 0 && last_commit >= 0)  // MMAs finished before the stages and TMEM go away
      if (!mbar_wait(sa_of(stage_bar + last_commit % kPStages), (uint32_t)((last_commit / kPStages) & 1),
                     kPWaitLimit))
        sh_pab = 1;
  } else {
    // ---- epilogue: one accumulator row per thread ----
    const int et = tid - 256, quarter = warp & 3, row = quarter * 32 + lane;
    for (int ti = 0, tile = blockIdx.x; tile < count; tile += gridDim.x, ++ti) {
      const TileItem it = items[tile];
      const SnMeta m = a.meta[it.s];
      const int acc = ti & 1;
      int64_t* cbase = maps + acc * 256;
      int64_t* crel = cbase + 128;
      if (it.mode == 1 && et < it.ncols) {
        const int jc = it.b_row0 + et;
        const RelGroup gr = a.groups[a.row_group[m.lidx + jc]];
        const SnMeta mt = a.meta[gr.t];
        cbase[et] = mt.off + (int64_t)(a.rows[m.lidx + jc] - mt.fc) * mt.ld;
        crel[et] = gr.rel_off - gr.j0;
      }
      if (et == 0) sh_eok[acc] = mbar_wait(sa_of(full_bar + acc), (uint32_t)((ti >> 1) & 1), kPWaitLimit) ? 1 : 0;
      named_sync(2, 128);  // maps ready; the accumulator is full (or the wait gave up)
      if (!sh_eok[acc]) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      float* L = static_cast<float*>(a.L);
      const int jr = it.a_row0 + row;
      int64_t last = INT64_MIN;
      int pos = 0;
      for (int c0 = 0; c0 < kUN; c0 += 32) {
        uint32_t v[32];
        const uint32_t taddr = tmem + (uint32_t)(acc * kUTmemCols) + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
              "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
              "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
              "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (row < it.mrows) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int c = c0 + j, jc = it.b_row0 + c;
            if (c < it.ncols && jr >= jc) {
              const float val = -__uint_as_float(v[j]);
              if (it.mode == 0) {
                atomicAdd(L + m.off + jr + (int64_t)jc * m.ld, val);
              } else {
                const int64_t cr = crel[c];
                if (cr != last) {
                  pos = a.rel[cr + jr];
                  last = cr;
                }
                atomicAdd(L + cbase[c] + pos, val);
              }
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(sa_of(empty_bar + acc)) : "memory");
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if ((sh_pab || !sh_eok[0] || !sh_eok[1]) && tid == 0) report_status(a.status, 3, -1, -1);
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(2 * kUTmemCols)
                 : "memory");
  }
}

}  // namespace

static int g_sms = 148;  // persistent tile grid: one CTA per SM
static int g_fper64 = 1, g_fper32 = 1;  // resident CTAs per SM of the persistent factorization

// ---- persistent factorization ------------------------------------------------------
// One CTA per SM takes the tasks of Plan::ftasks in order from an atomic counter,
// waits until the counters it depends on reach their targets (thread 0 polls with
// acquire loads, bounded), runs the task body with the whole block and publishes with
// release reductions on the counters it bumps.  The order is topological, so every
// task a CTA waits for was handed out earlier to a running CTA.
namespace {

__device__ __forceinline__ int ld_acquire_i(const int32_t* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_i(int32_t* p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int status_of(const Status* st) { return *(volatile const int32_t*)&st->code; }
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned smid() {
  unsigned r;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
  return r;
}

// The largest task body: the DMMA tile (FP64), the TMA-fed tcgen05 tile (FP32), whose
// stages and barriers sit above every other body's shared memory (at most 96 KB).
constexpr size_t kFSmemBytes = kDSmemBytes;  // the DMMA pipe and its barriers (above every other body's)
static_assert(kFSmemBytes >= 96 * 1024 + DTile<kDTileN>::kIntsBytes + 2 * kDStages * sizeof(uint64_t),
              "small panels (96 KB) stay below the DMMA stage barriers");
constexpr size_t kFSmemBytes32 = kVSmemBytes;
static_assert(kFSmemBytes32 >= 96 * 1024 + 1024, "FP32 persistent shared memory");

// FP64: two CTAs per SM (128 x 64 DMMA tiles); FP32: one (the TMA-fed tile's 193 KB).
template <class T>
__global__ void __launch_bounds__(256, std::is_same<T, float>::value ? 1 : 2)
    k_factor_persistent(FactorArgs a, FactorSched f) {
  constexpr bool kF32 = std::is_same<T, float>::value;
  extern __shared__ __align__(16) unsigned char smem_f[];
  __shared__ int sh_task, sh_go;
  TcTile tc;
  DmPipe dp;
  if constexpr (kF32) tc_setup(tc, smem_f);  // tensor memory and stage barriers for the whole launch
  else dm_setup<kDTileN>(dp, smem_f);
  for (;;) {
    if (threadIdx.x == 0) {
      int tk = atomicAdd(f.counter, 1);
      int go = tk < f.ntasks && status_of(a.status) == 0;
      if (go && f.trace) f.trace[4 * (size_t)tk] = global_ns();
      if (go) {
        const FTask t = f.tasks[tk];
        for (int w = 0; w < t.nwait && go; ++w) {
          const FWait fw = w == 0 ? FWait{t.w0_ctr, t.w0_target} : f.waits[t.wait0 + w];
          const int32_t* c = f.ctr + fw.ctr;
          if (ld_acquire_i(c) >= fw.target) continue;
          go = 0;
          for (long long it = 0; it < f.spin_limit; ++it) {
            if (it >= 256) __nanosleep(128);
            if (ld_acquire_i(c) >= fw.target) {
              go = 1;
              break;
            }
            if (status_of(a.status) != 0) break;
          }
          if (!go && atomicCAS(&a.status->code, 0, 3) == 0) {  // a wait expired
            a.status->supernode = -1;
            a.status->column = fw.ctr;
          }
        }
      }
      if (go && f.trace) {
        f.trace[4 * (size_t)tk + 1] = global_ns();
        f.trace[4 * (size_t)tk + 3] = smid();
      }
      sh_task = tk;
      sh_go = go;
    }
    __syncthreads();
    const int tk = sh_task;
    if (!sh_go) break;
    const FTask t = f.tasks[tk];
    switch (t.kind) {
      case 0:
        ftask::factor_small_task<T>(a, f.small_items[t.item], reinterpret_cast<double*>(smem_f));
        break;
      case 1:
        if (!kF32 && a.ldl) ftask::ldl_diag_task<T>(a, f.panel[t.item], f.winv, reinterpret_cast<double*>(smem_f));
        else ftask::potrf_diag_task<T>(a, f.panel[t.item], f.winv, reinterpret_cast<double*>(smem_f));
        break;
      case 2:
        ftask::trsm_rows_task<T>(a, f.panel[t.item], f.winv, reinterpret_cast<double*>(smem_f));
        break;
      case 3:
        simt_tile_task<T>(a, f.tiles[t.item], smem_f);
        break;
      default:
        if constexpr (kF32) tc32t_tile_task(a, f.tiles[t.item], tc);  // a failure records status 3
        else dmma_tile_task<kDTileN>(a, f.tiles[t.item], smem_f, dp);
        break;
    }
    __syncthreads();
    if (f.trace && threadIdx.x == 0) f.trace[4 * (size_t)tk + 2] = global_ns();
    for (int i = threadIdx.x; i < t.nsig; i += blockDim.x) red_release_i(f.ctr + f.sigs[t.sig0 + i], 1);
  }
  if constexpr (kF32) tc_teardown(tc);
}

}  // namespace

void launch_factor_persistent(cudaStream_t st, const FactorArgs& a, const FactorSched& f) {
  if (f.ntasks <= 0 || f.spin_limit <= 0) return;
  // as many CTAs as fit at once (a CTA only waits for tasks handed out before its own,
  // so the grid size is a matter of speed, not of progress)
  const int fit = (a.fp32 ? g_fper32 : g_fper64) * g_sms;
  const int grid = fit < f.ntasks ? fit : f.ntasks;
  if (a.fp32) k_factor_persistent<float><<<grid, 256, kFSmemBytes32, st>>>(a, f);
  else k_factor_persistent<double><<<grid, 256, kFSmemBytes, st>>>(a, f);
}

void init_gemm_attributes() {
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
  if (g_sms <= 0) g_sms = 148;
  cudaFuncSetAttribute(k_gemm_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTSmemBytes);
  cudaFuncSetAttribute(k_gemm_tc32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUSmemBytes);
  cudaFuncSetAttribute(k_gemm_tc32w, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWSmemBytes);
  cudaFuncSetAttribute(k_gemm_tc32p, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPSmemBytes);
  cudaFuncSetAttribute(k_gemm_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDSmemBytes);
  cudaFuncSetAttribute(k_factor_persistent<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFSmemBytes);
  cudaFuncSetAttribute(k_factor_persistent<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFSmemBytes32);
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_factor_persistent<double>, 256, kFSmemBytes) ==
          cudaSuccess &&
      nb > 0)
    g_fper64 = nb;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_factor_persistent<float>, 256, kFSmemBytes32) ==
          cudaSuccess &&
      nb > 0)
    g_fper32 = nb;
  cudaGetLastError();
}

void launch_gemm(cudaStream_t st, const FactorArgs& a, const TileItem* items, int count, int tile) {
  if (count <= 0) return;
  if (a.fp32) {
    if (tile == 128 && a.engine == 2)
      k_gemm_tc32p<<<count < g_sms ? count : g_sms, kPThreads, kPSmemBytes, st>>>(a, items, count);
    else if (tile == 128 && a.engine == 0) k_gemm_tc32<<<count, 256, kUSmemBytes, st>>>(a, items);
    else if (tile == 128 && a.engine == 3)
      k_gemm_tc32w<<<count < g_sms ? count : g_sms, kWThreads, kWSmemBytes, st>>>(a, items, count);
    else if (tile == 128) k_gemm_tf32x3<<<count, 256, kTSmemBytes, st>>>(a, items);
    else k_gemm_simt<float><<<count, 256, kSSmemBytes, st>>>(a, items);
  } else {
    if (tile == 128) k_gemm_dmma<<<count, kDThreads, kDSmemBytes, st>>>(a, items);
    else k_gemm_simt<double><<<count, 256, kSSmemBytes, st>>>(a, items);
  }
}

}  // namespace dev
}  // namespace spb
