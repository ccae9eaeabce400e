// Device kernels of the supernodal Cholesky factor and solve (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "plan.hpp"

namespace spb {
namespace dev {

// Status word shared by all kernels of one handle.  The first failure wins.
struct Status {
  int32_t code;        // 0 ok, 1 not SPD, 2 structure error, 3 device wait timed out
  int32_t supernode;   // 0-based supernode of the failing pivot
  int32_t column;      // 0-based permuted column of the failing pivot
  int32_t pad;
};

// Arguments shared by the factor kernels.
struct FactorArgs {
  void* L;                   // factor arena: double, or float when fp32
  const SnMeta* meta;        // nsuper
  const int32_t* rows;       // concatenated 0-based row lists
  const int32_t* supmember;  // 0-based supernode of each permuted column
  Status* status;
  const int32_t* row_group;  // relative-index group of each row-list entry
  const RelGroup* groups;
  const int32_t* rel;        // positions of update rows in their targets' row lists
  bool fp32;                 // FP32 factor storage (precision form)
  int engine;                // FP32 128 x 128 tiles: 0 tcgen05 per tile, 1 mma.sync, 2 persistent tcgen05,
                             // 3 tcgen05 fed by TMA
  // engine 3: split copies of the FP32 panels that have 128 x 128 tiles (per supernode
  // its offset in floats, -1 for none: hi rows then lo rows, row pitch round_up(w, 4)),
  // written by the tasks that finish panel rows, and their tiled tensor maps
  // (CUtensorMap, 128 B each, 64-byte aligned; map index per supernode)
  float* split = nullptr;
  const int64_t* split_off = nullptr;
  const void* tmaps = nullptr;
  const int32_t* tmap_of = nullptr;
  // LDL^T (FP64 only): L holds the unit factor (1 on the diagonal) and the working
  // matrix of unfactored columns; W (same layout) holds L D, so that its diagonal
  // is D.  Updates are C = L_a (L_b D)^T: the second operand is read from W.
  bool ldl;
  double* W;
};

// Doubles per diagonal-block scratch slot (see launch_potrf_diag).
constexpr size_t kDiagSlotDoubles = 64 * 64 + 128;

// Must run once per process (per device) before the first launch or capture.
void init_kernel_attributes();
void init_gemm_attributes();
void launch_assemble(cudaStream_t st, void* L, bool fp32, const int64_t* dst, const double* vals, int64_t nnz);
void launch_factor_small(cudaStream_t st, const FactorArgs& a, const int32_t* items, int count, int smem_bytes);
// winv: scratch of (diagonal blocks per step) x (64 x 64 + 128) doubles: factored block, 1/L_kk
// and (LDL^T) 1/D_kk
void launch_potrf_diag(cudaStream_t st, const FactorArgs& a, const PanelItem* items, int count, double* winv);
void launch_trsm_rows(cudaStream_t st, const FactorArgs& a, const PanelItem* items, int count, const double* winv);
// tile 64: FMA tiles (FP64 or FP32); tile 128: tensor-core tiles (FP64 DMMA, or 3xTF32 for FP32)
void launch_gemm(cudaStream_t st, const FactorArgs& a, const TileItem* items, int count, int tile);

// Persistent factorization (FP64, Cholesky or LDL^T): one launch runs every task of
// Plan::ftasks; ctr (Plan::nfctr) and counter must be zero at launch.  Waits are
// bounded by spin_limit polls (~128 ns apart); on expiry status 3 is recorded and every
// CTA leaves.
struct FactorSched {
  const FTask* tasks;
  int ntasks;
  const FWait* waits;
  const int32_t* sigs;
  int32_t* ctr;
  int32_t* counter;  // next task to hand out
  const int32_t* small_items;
  const PanelItem* panel;
  const TileItem* tiles;
  double* winv;      // scratch slots of the diagonal blocks
  long long spin_limit;
  unsigned long long* trace;  // optional, 4 per task: grabbed, dependencies met, done (ns), SM id
};
void launch_factor_persistent(cudaStream_t st, const FactorArgs& a, const FactorSched& f);

// Solves work on the permuted right-hand sides X (n x nrhs, column-major, leading dimension ldx).

// Persistent sweeps (one launch each).  counter, arrived, blkdone and upd must
// be zero at launch; expected[s] is the number of forward arrivals (off-diagonal
// task, target) that write rows of supernode s.  Forward: Y = X (accumulated),
// solution to Z; backward: Z (accumulated), solution to X.
struct PSolveArgs {
  const void* L;     // factor arena (double, or float when fp32): L, or L D for the LDL^T forward sweep
  const void* Inv;   // diagonal super-block inverses of that operand (same type)
  bool fp32;
  const SnMeta* meta;
  const int32_t* rows;
  const int32_t* supmember;
  const int32_t* sparent;
  const int32_t* row_group;  // relative-index group of each row-list entry (arrival targets)
  const RelGroup* groups;
  double* X;
  double* Z;
  int64_t ldx;       // leading dimension of X and Z
  int nrhs;  // <= 64
  const SolveTask* tasks;
  int ntasks;
  const int32_t* tiny;  // leaf supernodes of the forward T tasks (Plan::tiny)
  int32_t* counter;
  const int32_t* expected;
  int32_t* arrived;
  int32_t* blkdone;  // per supernode: finished diagonal tasks of this sweep
  int32_t* upd;      // per super-block (meta.sboff + p): updates landed
  int sb;            // 64-column blocks per super-block (Plan::solve_sb)
  int tpt;           // tiles per DI / U / V / O / W task (Plan::solve_tpt)
  Status* status;
  long long spin_limit;  // polls (about 128 ns apart) before a wait gives up
  unsigned long long* trace;  // optional, 4 per task: grabbed, dependencies met, done (ns), s << 8 | kind
};
void init_solve_attributes();
void launch_solve_persistent(cudaStream_t st, const PSolveArgs& a, bool forward);
// Inverses of the diagonal super-blocks of L (the whole list of items, Plan::inv_items),
// written to Inv in 64 x 64 tiles at meta.ioff.
void launch_sb_inverse(cudaStream_t st, const void* L, void* Inv, bool fp32, const SnMeta* meta,
                       const InvItem* items, int count, int sb);

// Precision form (FP64 refinement): gather CSR values, residual r = b - A x,
// per-column max |v| (out zeroed by the caller), max row sum of |A|, x += d.
void launch_gather(cudaStream_t st, double* dst, const double* src, const int64_t* idx, int64_t n);
void launch_residual(cudaStream_t st, const int64_t* rowptr, const int32_t* col, const double* val, const double* x,
                     const double* b, double* r, int n, int nrhs, int64_t ld);
void launch_segmax(cudaStream_t st, const double* v, int n, int nrhs, int64_t ld, const int32_t* rowseg,
                   double* out);
void launch_rowsum_segmax(cudaStream_t st, const int64_t* rowptr, const double* val, int n, const int32_t* rowseg,
                          double* anorm);
void launch_eta(cudaStream_t st, const double* anorm, const double* bmax, const double* xmax, const double* rmax,
                int nseg, int nrhs, double* eta);
void launch_axpy(cudaStream_t st, double* x, const double* d, int n, int nrhs, int64_t ld);

// X[invp[i], c] = B[i, c]   and   B[i, c] = X[invp[i], c]
void launch_permute_in(cudaStream_t st, double* X, int64_t ldx, const double* B, int64_t ldb,
                       const int32_t* invp0, int n, int nrhs);
void launch_permute_out(cudaStream_t st, double* B, int64_t ldb, const double* X, int64_t ldx,
                        const int32_t* invp0, int n, int nrhs);

}  // namespace dev
}  // namespace spb
