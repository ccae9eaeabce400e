// Device plan: how the supernodal factor is laid out in HBM and in which order
// the hot-path kernels visit it.  Built once per sparsity structure on the host
// from the symbolic result; reused by every numeric factorization and solve.
//
// Layout.  Supernode s owns one column-major panel of h_s x w_s doubles (the
// diagonal block followed by every off-diagonal row of its structure), with a
// leading dimension ld_s >= h_s padded to a multiple of 4 and a panel offset
// that is a multiple of 32 elements (256 B).  This is the reference's set of
// cells (K, s) (symPACKMatrix2D.hpp:499-944) stored contiguously: cell (K, s)
// is the run of panel rows whose global row falls in supernode K.
//
// Schedule.  The supernodal elimination tree is levelled by height (leaves at
// level 0).  Supernodes of one level never depend on each other, so one level
// is: factor all of its panels, then scatter all of their Schur-complement
// updates into ancestors.  This is the reference's FACTOR -> TRSM ->
// UPDATE2D_COMP dependency chain (symPACKMatrix2D.hpp:3893-3997) collapsed to
// supernode granularity.
#pragma once
#include <cstdint>
#include <vector>

#include "symbolic.hpp"

namespace spb {

// Panel descriptor (device-visible).
struct SnMeta {
  int32_t fc;    // first column, 0-based (permuted numbering)
  int32_t w;     // width (number of columns)
  int32_t h;     // rows, including the w x w diagonal block
  int32_t ld;    // leading dimension of the panel
  int64_t off;   // element offset of the panel in the factor arena
  int64_t lidx;  // offset of this supernode's row list in the device row array
  int32_t boff;  // first of this supernode's 64-column blocks over all supernodes
  int32_t sboff; // first of this supernode's solve super-blocks in the per-super-block solve counters
  int64_t ioff;  // element offset of its diagonal super-block inverses in the inverse arena (-1: none)
};

// One tile of a Schur-complement product  C = A * B^T  over panel columns
// [k0, k0+kn) of supernode s, rows a_row0.. of A and b_row0.. of B (panel rows).
//  mode 0: in-panel update, C is subtracted from panel(s) rows a_row0+i, columns b_row0+j
//  mode 1: external update, C is scatter-subtracted into the ancestors that own
//          global rows lindx_s[a_row0+i] x lindx_s[b_row0+j]
struct TileItem {
  int32_t s;
  int32_t mode;
  int32_t a_row0;
  int32_t b_row0;
  int32_t k0;
  int32_t kn;
  int32_t mrows;  // valid rows in this tile (<= tile height)
  int32_t ncols;  // valid columns in this tile (<= tile width)
};

// One launch of the factorization sequence.
enum class StepKind : int32_t {
  FactorSmall = 0,   // fused POTRF + TRSM of whole panels in shared memory (items = supernode ids)
  PotrfDiag = 1,     // POTRF of one 64-column diagonal block of a wide panel (PanelItem, row0 = -1)
  TrsmRows = 2,      // TRSM of 64-row tiles below that block (PanelItem)
  Gemm = 3,          // TileItem list (in-panel or external update)
};
// Stream lanes of the captured factorization (look-ahead): the chain of a
// level's wide panels (POTRF, TRSM and the update of the next column tile) runs
// in order on the main stream; the update of the remaining columns of block k
// runs on a side stream beside the chain and must finish before the POTRF of
// block k + 2; a join step (small panels, external updates) waits for all side work.
enum class Lane : int32_t { Chain = 0, Side = 1, Join = 2 };

struct Step {
  StepKind kind;
  int32_t begin;  // range into the matching item array
  int32_t count;
  int32_t arg;    // PotrfDiag/TrsmRows: column block start c0; FactorSmall: shared-memory bytes
  int32_t tile;   // Gemm: tile edge (64 or 128)
  Lane lane = Lane::Join;
  int32_t blk = 0;  // Chain / Side: column block index k = c0 / 64
};

// Panel-block work: supernode s, column block [c0, c0+nb), row tile starting at row0.
struct PanelItem {
  int32_t s;
  int32_t c0;
  int32_t nb;
  int32_t row0;   // first panel row of the row tile (>= c0+nb); -1 for the diagonal block
  int32_t slot;   // scratch slot holding this step's L11^-1 for the supernode
};

// One task of the persistent factorization: a small panel, a diagonal block, a TRSM
// row tile or an update tile (the items of the step sequence), with the dependency
// counters it waits for and the ones it bumps when done.  Counters: per supernode the
// external update tiles landed (ext) and its finished panel tasks (sdone), per 64-column
// block its finished POTRF / TRSM tasks (blk) and the in-panel update tiles landed in
// its columns (col).
struct FTask {
  int32_t kind;   // 0 small panel, 1 diagonal block, 2 TRSM row tile, 3 64 x 64 tile, 4 128 x 128 tile
  int32_t item;   // index into small_items / panel_items / tile_items
  int32_t wait0;  // fwaits[wait0 .. wait0 + nwait)
  int32_t nwait;
  int32_t sig0;   // fsigs[sig0 .. sig0 + nsig)
  int32_t nsig;
  int32_t w0_ctr;     // copy of the first wait, fwaits[wait0] (when nwait > 0), so that
  int32_t w0_target;  // dispatch reads it with the task instead of after it
};
struct FWait {
  int32_t ctr;
  int32_t target;
};

// One task of the persistent triangular solves.  A supernode of one 64-column block
// is solved by substitution; a wider one is cut into super-blocks of sb 64-column
// blocks (the last one shorter), and the diagonal triangle of every super-block p is
// applied through its inverse Inv_p (computed once per factorization, in 64 x 64
// tiles), so a super-block costs two parallel steps instead of a chain of sb block
// solves.  Forward (permuted right-hand sides Y in, solution of L y = b in Z):
//            kind 6  T(i, t):  t tiny leaf supernodes tiny[i .. i + t), one per thread, whole
//                              (no arrivals to wait for; solve, scatter, signal)
//            kind 4  F:        one-block supernode with at most kSolveFusedTiles
//                              off-diagonal tiles, whole: Z_0 <- L_00^-1 Y_0, then every
//                              tile's Y[ancestor rows] -= L_u0 Z_0
//            kind 0  D:        one-block supernode: Z_0 <- L_00^-1 Y_0
//            kind 5  DI(p, r): Z[block r of p] <- sum_{q <= r} Inv_p(r, q) Y[block q of p]
//                              once the descendants' and earlier super-blocks' updates landed
//            kind 1  U(p, t):  Y[block t] -= L(t, super-block p) Z[p]   (t in a later super-block)
//            kind 2  O(p, u):  Y[rows of off-diagonal tile u] -= L(u, super-block p) Z[p],
//                              scattered into the ancestors' rows
// Backward (Z in, solution X):
//            kind 6  T(i, t):  the tiny leaves, one per thread, each once its parent is done
//            kind 4  G:        the F supernode whole: Z_0 -= L_u0^T X[ancestor rows of u] for
//                              every tile, then X_0 <- L_00^-T Z_0
//            kind 3  W(p, u):  Z[p] -= L(u, super-block p)^T X[ancestor rows of tile u]
//                              (final once the parent is done)
//            kind 0  B:        one-block supernode: X_0 <- L_00^-T Z_0
//            kind 5  DI(p, r): X[block r of p] <- sum_{q >= r} Inv_p(q, r)^T Z[block q of p]
//            kind 1  V(p, t):  Z[block t] -= L(super-block p, t)^T X[p]   (t in an earlier super-block)
// Task lists are topological: every task a task waits on comes earlier.
// DI, U, V, O and W tasks each cover at most tpt of their 64 x 64 tiles (the first one
// q0), adding their part atomically, so that a step of a wide supernode's chain is
// spread over many CTAs.
struct SolveTask {
  int32_t s;
  int32_t kind;
  int32_t i;  // super-block p (DI, U, V, O, W) | first tile q0 << 24
  int32_t t;  // block r within p (DI), target block t (U, V) or tile u (O, W)
};
inline int32_t pack_task_i(int p, int q0) { return p | (q0 << 24); }

// Task counts of the super-block solve (host and device): tasks of a run of `tiles`
// tiles, and the DI tasks of a super-block of nb blocks (sum over its rows r of the
// tasks of r + 1 tiles; the same sum counts the backward rows of nb - r tiles).
#ifdef __CUDACC__
#define SPB_HD __host__ __device__
#else
#define SPB_HD
#endif
SPB_HD inline int solve_ntask(int tiles, int tpt) { return (tiles + tpt - 1) / tpt; }
SPB_HD inline int solve_di_tasks(int nb, int tpt) {
  int c = 0;
  for (int r = 0; r < nb; ++r) c += solve_ntask(r + 1, tpt);
  return c;
}
// DI tasks of super-blocks p0 .. p1 - 1 of a supernode of nblk blocks.
SPB_HD inline int solve_di_range(int nblk, int sb, int tpt, int p0, int p1) {
  const int nsb = (nblk + sb - 1) / sb, nlast = nblk - (nsb - 1) * sb;
  int c = 0;
  for (int p = p0; p < p1; ++p) c += solve_di_tasks(p == nsb - 1 ? nlast : sb, tpt);
  return c;
}
// Diagonal tasks that mark a supernode done in a sweep (the count its blkdone reaches).
SPB_HD inline int solve_done_count(int w, int sb, int tpt) {
  const int nblk = (w + 63) / 64;
  return nblk == 1 ? 1 : solve_di_range(nblk, sb, tpt, 0, (nblk + sb - 1) / sb);
}

// One CTA of the super-block inverse kernel: column block j of Inv_p of supernode s
// (tiles (i, j), i = j .. nb_p - 1).
struct InvItem {
  int32_t s;
  int32_t p;
  int32_t j;
  int32_t pad;
};

// 64 x 64 tiles of the inverse of a super-block of nb blocks (lower triangle of tiles).
inline int64_t inv_tiles(int nb) { return (int64_t)nb * (nb + 1) / 2; }

// Relative indices of the external updates (the src_to_tgt_offset maps of
// symPACKMatrix2D.hpp:1395-1466, computed once per structure instead of per
// update).  The off-diagonal rows of supernode s that fall in ancestor t form
// one group; for every off-diagonal row r of s at or after the group's first
// row j0, rel[rel_off + (r - j0)] is the position of that row in t's row list.
struct RelGroup {
  int32_t t;        // target supernode (0-based)
  int32_t j0;       // panel row of s where the group starts (>= w)
  int64_t rel_off;  // offset of the group's positions in the rel array
};

struct Plan {
  int n = 0;
  int nsuper = 0;
  int nlevels = 0;
  int64_t arena_elems = 0;      // total doubles in the factor arena
  int64_t lindx_total = 0;
  std::vector<SnMeta> meta;     // nsuper
  std::vector<int32_t> rows;    // concatenated 0-based row lists (device copy)
  std::vector<int32_t> row_group;   // per row-list entry: its RelGroup (off-diagonal rows), else -1
  std::vector<RelGroup> groups;
  std::vector<int32_t> rel;         // positions in the target row lists
  std::vector<int32_t> supmember0;  // 0-based supernode of each (permuted) column
  std::vector<int32_t> sparent;     // supernodal etree parent (0-based, -1 root)
  std::vector<int32_t> level;       // height level of each supernode
  std::vector<std::vector<int32_t>> level_sn;  // supernodes per level
  // factorization sequence
  std::vector<int32_t> small_items;  // supernode ids for FactorSmall steps
  std::vector<PanelItem> panel_items;
  std::vector<TileItem> tile_items;
  std::vector<Step> steps;
  int32_t max_diag_slots = 0;      // scratch slots of the diagonal blocks (one per diagonal block)
  // persistent factorization: tasks in dispatch order (topological), their waits and signals
  std::vector<FTask> ftasks;
  std::vector<FWait> fwaits;
  std::vector<int32_t> fsigs;
  int32_t nfctr = 0;               // counters: ext[ns], sdone[ns], blk[nblk_total], col[nblk_total]
  double fsim_us = 0.0;            // makespan of the list-scheduling simulation that ordered them
  std::vector<double> step_flops;  // useful (algorithmic) flops of each step
  // executed flop count of the sequence (w^3/3 + m w^2 + m^2 w per supernode)
  double exec_flops = 0.0;
  std::vector<uint8_t> is_big;
  // persistent solves: forward tasks (postorder), backward tasks (reverse),
  // and per supernode the number of forward off-diagonal tiles writing its rows
  std::vector<SolveTask> fwd_tasks, bwd_tasks;
  std::vector<int32_t> fwd_pending;
  std::vector<int32_t> tiny;  // leaf supernodes of the forward T tasks
  int32_t nblk_total = 0;  // 64-column blocks over all supernodes
  int32_t nsb_total = 0;   // solve super-blocks over all supernodes (per-super-block counters)
  int32_t solve_sb = 8;    // 64-column blocks per solve super-block
  int32_t solve_tpt = 2;   // 64 x 64 tiles per DI / U / V / O / W task
  // diagonal super-block inverses: arena size (elements) and one item per (super-block, column block)
  int64_t inv_elems = 0;
  std::vector<InvItem> inv_items;
  // algorithmic bytes of one sweep: every panel element read once
  double solve_sweep_bytes = 0.0;
};

// Supernodes of one 64-column block with at most this many off-diagonal 64-row tiles
// are one solve task per sweep.
constexpr int kSolveFusedTiles = 16;
// Tiny leaf supernodes (at most kTinyMaxW columns and kTinyMaxElems panel entries) are
// solved forward one per thread, kTinyBatch to a task.
constexpr int kTinyMaxW = 4, kTinyMaxElems = 64, kTinyBatch = 128;

// Tunables of the plan.
struct PlanParams {
  int small_max_w = 32;          // widest panel handled by the fused small-panel kernel
  int small_max_bytes = 96 * 1024;
  int nb = 64;                   // column block of the blocked panel factorization
  int outer_nb = 256;            // outer block: the trailing columns are updated once per outer block
  int big_tile_rows = 128;       // products with at least this many rows use 128 x 128 tensor-core tiles
  int solve_sb = 8;              // 64-column blocks per solve super-block (>= 1)
  int solve_tpt = 2;             // 64 x 64 tiles per DI / U / V / O / W solve task (>= 1)
  int sms = 148;                 // SMs of the device: a launch with too few tiles to fill them
                                 // splits its tiles' K range (partial products add atomically)
  bool factor_dag = true;        // build the persistent factorization's task graph (FP64 handles)
  bool fp32 = false;             // FP32 factor (precision form): 128 x 128 tensor-core tiles, one CTA
                                 // per SM; FP64: 128 x 64 tiles at two CTAs per SM
  bool operator==(const PlanParams& o) const {
    return small_max_w == o.small_max_w && small_max_bytes == o.small_max_bytes && nb == o.nb &&
           outer_nb == o.outer_nb && big_tile_rows == o.big_tile_rows && solve_sb == o.solve_sb &&
           solve_tpt == o.solve_tpt && sms == o.sms && factor_dag == o.factor_dag && fp32 == o.fp32;
  }
};

Plan build_plan(const Symbolic& s, const PlanParams& p = PlanParams());

// Re-order the persistent factorization's tasks (P.ftasks, fwaits, fsigs, fsim_us) by the
// same list scheduling with measured durations in place of the cost model: us[i] is the
// duration of task P.ftasks[i] in microseconds (<= 0 keeps the model's estimate).  The
// counts of tasks, waits and signals do not change; the dependency counters neither.
void reorder_factor_tasks(Plan& P, const PlanParams& prm, const std::vector<double>& us);

// int32 counters one persistent solve pass uses: two task counters, then per
// supernode arrivals and forward / backward done blocks, then per super-block
// forward / backward update counts.  Sized by 64-column blocks (at least as many
// as super-blocks).
inline size_t solve_sync_ints(const Plan& P) { return 2 + 3 * (size_t)P.nsuper + 2 * (size_t)P.nblk_total; }

// Destination of each entry of A's lower triangle (input order) in the arena,
// DistributeMatrix (symPACKMatrix2D.hpp:6336-6576) done once per structure.
std::vector<int64_t> build_assembly_map(const Symbolic& s, const Plan& plan, const int64_t* colptr,
                                        const int32_t* rowind);

}  // namespace spb
