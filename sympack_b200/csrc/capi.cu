// extern "C" boundary of the supernodal Cholesky path (declared in
// include/sympack_b200.h).  A handle plays the role of one symPACKMatrix2D
// object at one rank: it owns the symbolic analysis (host), the device plan,
// the factor arena in HBM, and a CUDA graph replaying the factorization.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <atomic>
#include <mutex>
#include <thread>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sympack_b200.h"
#include "kernels.cuh"
#include "plan.hpp"
#include "symbolic.hpp"

using spb::dev::Status;

struct spb_handle {
  spb_options opt{};
  int device = 0;
  cudaStream_t stream = nullptr;      // stream every call runs on
  cudaStream_t own_stream = nullptr;  // created by spb_create
  cudaStream_t side_stream = nullptr; // look-ahead updates of the captured factorization
  std::vector<cudaEvent_t> lane_events;
  std::string err;
  bool have_symbolic = false, have_values = false, factored = false, have_solution = false;
  spb::Symbolic sym;
  spb::Plan plan;
  spb::Cells cells;
  bool cells_built = false;
  int64_t nnz_a = 0;
  std::vector<int64_t> colptr;
  std::vector<int32_t> rowind;
  std::vector<int64_t> amap;       // arena position of each input entry (DistributeMatrix map)
  std::vector<int32_t> level_off;  // level l covers dlevel_sn[level_off[l] .. level_off[l+1])
  // device buffers
  bool fp32 = false;        // precision form: FP32 factor + FP64 refinement
  bool ldl = false;         // LDL^T decomposition (FP64): dL unit L, dW = L D
  size_t elem = 8;          // bytes per factor entry
  void* dL = nullptr;
  double* dW = nullptr;
  spb::SnMeta* dmeta = nullptr;
  int32_t* drows = nullptr;
  int32_t* dsupm = nullptr;
  int32_t* drowgrp = nullptr;      // relative-index group of each row-list entry
  spb::RelGroup* dgroups = nullptr;
  int32_t* drel = nullptr;
  int64_t* damap = nullptr;
  double* dA = nullptr;
  int32_t* dsmall = nullptr;
  spb::PanelItem* dpanel = nullptr;
  double* dwinv = nullptr;  // factored diagonal blocks (FP64) and 1/L_kk of one step
  spb::TileItem* dtiles = nullptr;
  float* dsplit = nullptr;         // FP32 engine 3: split copies of the panels with 128 x 128 tiles
  int64_t* dsplit_off = nullptr;   // offset of each supernode's copy (-1: none)
  CUtensorMap* dtmaps = nullptr;   // their tiled tensor maps
  int32_t* dtmap_of = nullptr;     // map of each supernode (-1: none)
  spb::FTask* dftasks = nullptr;   // persistent factorization: tasks, waits, signals, counters
  spb::FWait* dfwaits = nullptr;
  int32_t* dfsigs = nullptr;
  int32_t* dfctr = nullptr;        // nfctr counters + the task counter
  unsigned long long* dftrace = nullptr;  // factor trace (spb_set_factor_trace): 4 per task
  bool factor_trace = false;
  bool trace_fresh = false;        // the last factorization was traced in the current task order
  int32_t* dinvp0 = nullptr;
  int32_t* dlevel_sn = nullptr;
  spb::SolveTask* dfwd = nullptr;
  spb::SolveTask* dbwd = nullptr;
  int32_t* dexpected = nullptr;
  int32_t* dtiny = nullptr;        // leaf supernodes of the forward sweep's T tasks
  int32_t* dsparent = nullptr;
  int32_t* dsync = nullptr;  // solve counters (spb::solve_sync_ints)
  void* dInv = nullptr;      // diagonal super-block inverses of the forward operand (L, or L D for LDL^T)
  void* dInvB = nullptr;     // LDL^T: inverses of the backward operand (unit L); else dInv
  spb::InvItem* dinvitems = nullptr;
  bool inv_stale = true;     // inverses not yet computed for the current factor
  Status* dstatus = nullptr;
  // precision form: original matrix as full CSR (FP64) and refinement buffers
  std::vector<int64_t> csr_rowptr;
  std::vector<int32_t> csr_col;
  std::vector<int64_t> csr_src;
  int64_t* d_rowptr = nullptr;
  int32_t* d_col = nullptr;
  int64_t* d_csrsrc = nullptr;
  double* d_val = nullptr;
  // refinement norms of every system: [eta, anorm[nseg], bmax[nseg*64], xmax[nseg*64], rmax[nseg*64]]
  double* d_norms = nullptr;
  std::vector<int32_t> seg_off{};  // systems of a batch (0-based row offsets); empty = one system
  int32_t* d_rowseg = nullptr;     // system of each row (batches only)
  double* dR = nullptr;       // residual / correction right-hand side (original order)
  double* dD = nullptr;       // correction (original order)
  double* dXo = nullptr;      // refined solution (original order)
  int ir_iterations = 0;
  double backward_error = -1.0;
  double* dX = nullptr;
  double* dZ = nullptr;  // solve: forward solution / backward right-hand side (permuted)
  double* dB = nullptr;
  int64_t x_cap = 0;  // doubles available in dX, dZ and dB
  int x_nrhs = 0;
  int64_t device_bytes = 0;
  cudaGraphExec_t fgraph = nullptr;
  std::vector<void*> allocs;
  // profiling: per-launch event pairs, per-kind totals of the last profiled call
  long long wait_limit = 1LL << 24;  // ~2 s of polling per device wait
  int stall_supernode = -1;          // test hook: extra expected arrival nobody delivers
  bool profiling = false;
  bool prof_inverse = false;  // the last profiled solve computed the super-block inverses
  unsigned long long* dtrace = nullptr;  // profiled solves: 4 per task of each sweep (forward, backward)
  spb_profile prof{};
  std::vector<cudaEvent_t> events;
  // footprint predictions for the other precision: its plan, built on first use
  mutable std::mutex pred_mu;
  mutable std::unique_ptr<spb::Plan> pred_plan[2];
  mutable spb::PlanParams pred_prm[2];
};

namespace {

int fail(spb_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int cuda_fail(spb_handle* h, cudaError_t e, const char* what) {
  std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();
  return fail(h, e == cudaErrorMemoryAllocation ? SPB_ERR_OOM : SPB_ERR_CUDA, msg);
}

#define SPB_CK(h, call)                                   \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) return cuda_fail(h, _e, #call); \
  } while (0)

template <class T>
cudaError_t dalloc(spb_handle* h, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  // stream-ordered allocation: allocating or freeing one handle's buffers does
  // not synchronise the device, so handles served side by side keep running
  cudaError_t e = cudaMallocAsync((void**)p, count * sizeof(T), h->own_stream);
  if (e == cudaSuccess) {
    h->allocs.push_back((void*)*p);
    h->device_bytes += (int64_t)(count * sizeof(T));
  }
  return e;
}

void release_device(spb_handle* h) {
  if (h->fgraph) {
    cudaGraphExecDestroy(h->fgraph);
    h->fgraph = nullptr;
  }
  if (!h->allocs.empty()) {
    cudaStreamSynchronize(h->stream);  // work using the buffers has finished
    for (void* p : h->allocs) cudaFreeAsync(p, h->own_stream);
    cudaStreamSynchronize(h->own_stream);
  }
  h->allocs.clear();
  h->device_bytes = 0;
  h->dL = nullptr;
  h->dW = nullptr;
  h->dX = h->dZ = h->dB = h->dR = h->dD = h->dXo = nullptr;
  h->dInv = h->dInvB = nullptr;
  h->dsplit = nullptr;
  h->dsplit_off = nullptr;
  h->dtmaps = nullptr;
  h->dtmap_of = nullptr;
  h->dftrace = nullptr;
  h->d_rowseg = nullptr;
  h->dtrace = nullptr;
  h->x_cap = 0;
}

// The persistent factorization runs FP64 handles (unless the steps are asked for) and
// FP32 handles that ask for it and whose 128 x 128 tiles use the TMA-fed tcgen05 engine
// (the one with a task body for the persistent kernel).
bool persistent_schedule(const spb_options& o) {
  if (o.precision == SPB_PRECISION_FP64) return o.factor_schedule != SPB_FACTOR_STEPS;
  return o.factor_schedule == SPB_FACTOR_PERSISTENT && o.fp32_engine == 3;
}
bool persistent_factor(const spb_handle* h) { return persistent_schedule(h->opt); }

spb::dev::FactorArgs factor_args(spb_handle* h) {
  spb::dev::FactorArgs a;
  a.L = h->dL;
  a.meta = h->dmeta;
  a.rows = h->drows;
  a.supmember = h->dsupm;
  a.status = h->dstatus;
  a.row_group = h->drowgrp;
  a.groups = h->dgroups;
  a.rel = h->drel;
  a.fp32 = h->fp32;
  a.engine = h->opt.fp32_engine;
  a.split = h->dsplit;
  a.split_off = h->dsplit_off;
  a.tmaps = h->dtmaps;
  a.tmap_of = h->dtmap_of;
  a.ldl = h->ldl;
  a.W = h->dW;
  return a;
}

void launch_step(spb_handle* h, const spb::dev::FactorArgs& a, const spb::Step& st, cudaStream_t stream);

cudaEvent_t lane_event(spb_handle* h, size_t i) {
  while (h->lane_events.size() <= i) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
    h->lane_events.push_back(e);
  }
  return h->lane_events[i];
}

// Issue the factorization steps (captured into a graph).  Chain and join steps
// go to the handle's stream in order; side steps (the update of a block's
// remaining columns) go to the side stream after the chain has produced their
// operands, and the POTRF of block k waits for the side update of block k - 2,
// the last one that writes block k's columns.  Updates are atomic additions,
// so a chain update and a side update of the same columns may overlap.
cudaError_t enqueue_factor(spb_handle* h) {
  const spb::Plan& P = h->plan;
  spb::dev::FactorArgs a = factor_args(h);
  if (persistent_factor(h)) {  // every task in one launch, ordered by dependency counters
    spb::dev::FactorSched f{};
    f.tasks = h->dftasks;
    f.ntasks = (int)P.ftasks.size();
    f.waits = h->dfwaits;
    f.sigs = h->dfsigs;
    f.ctr = h->dfctr;
    f.counter = h->dfctr + P.nfctr;
    f.small_items = h->dsmall;
    f.panel = h->dpanel;
    f.tiles = h->dtiles;
    f.winv = h->dwinv;
    f.spin_limit = h->wait_limit;
    f.trace = h->factor_trace ? h->dftrace : nullptr;
    cudaMemsetAsync(h->dfctr, 0, sizeof(int32_t) * ((size_t)P.nfctr + 1), h->stream);
    spb::dev::launch_factor_persistent(h->stream, a, f);
    return cudaGetLastError();
  }
  size_t nev = 0;
  std::vector<std::pair<int, cudaEvent_t>> side;  // (block, event) of this level's side updates
  size_t waited = 0;                               // side events the chain already waits for
  bool pending = false;                            // side work not yet joined
  auto next_event = [&]() { return lane_event(h, nev++); };
  for (const spb::Step& st : P.steps) {
    if (st.lane == spb::Lane::Join) {
      if (pending) {
        cudaEvent_t e = next_event();
        if (!e) return cudaErrorMemoryAllocation;
        cudaEventRecord(e, h->side_stream);
        cudaStreamWaitEvent(h->stream, e, 0);
        pending = false;
      }
      side.clear();
      waited = 0;
      launch_step(h, a, st, h->stream);
    } else if (st.lane == spb::Lane::Chain) {
      if (st.kind == spb::StepKind::PotrfDiag) {
        size_t need = waited;
        while (need < side.size() && side[need].first <= st.blk - 2) ++need;
        if (need > waited) {
          cudaStreamWaitEvent(h->stream, side[need - 1].second, 0);
          waited = need;
        }
      }
      launch_step(h, a, st, h->stream);
    } else {
      cudaEvent_t fork = next_event(), done = next_event();
      if (!fork || !done) return cudaErrorMemoryAllocation;
      cudaEventRecord(fork, h->stream);
      cudaStreamWaitEvent(h->side_stream, fork, 0);
      launch_step(h, a, st, h->side_stream);
      cudaEventRecord(done, h->side_stream);
      side.emplace_back(st.blk, done);
      pending = true;
    }
  }
  if (pending) {
    cudaEvent_t e = next_event();
    if (!e) return cudaErrorMemoryAllocation;
    cudaEventRecord(e, h->side_stream);
    cudaStreamWaitEvent(h->stream, e, 0);
  }
  return cudaGetLastError();
}

void launch_step(spb_handle* h, const spb::dev::FactorArgs& a, const spb::Step& st, cudaStream_t stream) {
  {
    switch (st.kind) {
      case spb::StepKind::FactorSmall:
        spb::dev::launch_factor_small(stream, a, h->dsmall + st.begin, st.count, st.arg);
        break;
      case spb::StepKind::PotrfDiag:
        spb::dev::launch_potrf_diag(stream, a, h->dpanel + st.begin, st.count, h->dwinv);
        break;
      case spb::StepKind::TrsmRows:
        spb::dev::launch_trsm_rows(stream, a, h->dpanel + st.begin, st.count, h->dwinv);
        break;
      case spb::StepKind::Gemm:
        spb::dev::launch_gemm(stream, a, h->dtiles + st.begin, st.count, st.tile);
        break;
    }
  }
}

int check_handle(spb_handle* h) { return h ? SPB_OK : SPB_ERR_INVALID; }

int num_segments(const spb_handle* h) { return h->seg_off.empty() ? 1 : (int)h->seg_off.size() - 1; }

cudaError_t ensure_events(spb_handle* h, size_t count) {
  while (h->events.size() < count) {
    cudaEvent_t e;
    cudaError_t err = cudaEventCreate(&e);
    if (err != cudaSuccess) return err;
    h->events.push_back(e);
  }
  return cudaSuccess;
}

int step_kind(const spb::Step& st) {
  switch (st.kind) {
    case spb::StepKind::FactorSmall: return SPB_KIND_FACTOR_SMALL;
    case spb::StepKind::PotrfDiag: return SPB_KIND_POTRF_DIAG;
    case spb::StepKind::TrsmRows: return SPB_KIND_TRSM_ROWS;
    default: return st.tile == 128 ? SPB_KIND_GEMM_DMMA : SPB_KIND_GEMM_SIMT;
  }
}

void clear_kinds(spb_handle* h, int first, int last) {
  for (int k = first; k <= last; ++k) {
    h->prof.ms[k] = h->prof.flops[k] = h->prof.bytes[k] = 0.0;
    h->prof.launches[k] = 0;
  }
}

// Eager factorization with one event pair per launch (profiling mode).
int factor_profiled(spb_handle* h) {
  const spb::Plan& P = h->plan;
  SPB_CK(h, ensure_events(h, 2 * P.steps.size()));
  spb::dev::FactorArgs a = factor_args(h);
  for (size_t k = 0; k < P.steps.size(); ++k) {
    const spb::Step& st = P.steps[k];
    SPB_CK(h, cudaEventRecord(h->events[2 * k], h->stream));
    switch (st.kind) {
      case spb::StepKind::FactorSmall:
        spb::dev::launch_factor_small(h->stream, a, h->dsmall + st.begin, st.count, st.arg);
        break;
      case spb::StepKind::PotrfDiag:
        spb::dev::launch_potrf_diag(h->stream, a, h->dpanel + st.begin, st.count, h->dwinv);
        break;
      case spb::StepKind::TrsmRows:
        spb::dev::launch_trsm_rows(h->stream, a, h->dpanel + st.begin, st.count, h->dwinv);
        break;
      case spb::StepKind::Gemm:
        spb::dev::launch_gemm(h->stream, a, h->dtiles + st.begin, st.count, st.tile);
        break;
    }
    SPB_CK(h, cudaEventRecord(h->events[2 * k + 1], h->stream));
  }
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  clear_kinds(h, SPB_KIND_FACTOR_SMALL, SPB_KIND_GEMM_DMMA);
  for (size_t k = 0; k < P.steps.size(); ++k) {
    float ms = 0.f;
    SPB_CK(h, cudaEventElapsedTime(&ms, h->events[2 * k], h->events[2 * k + 1]));
    int kind = step_kind(P.steps[k]);
    h->prof.ms[kind] += ms;
    h->prof.flops[kind] += P.step_flops[k];
    h->prof.launches[kind] += 1;
  }
  return SPB_OK;
}

int ensure_rhs_capacity(spb_handle* h, int nrhs) {
  if (h->profiling && !h->dtrace) {  // task timeline of profiled solves
    SPB_CK(h, dalloc(h, &h->dtrace, 4 * (h->plan.fwd_tasks.size() + h->plan.bwd_tasks.size())));
    SPB_CK(h, cudaStreamSynchronize(h->own_stream));
  }
  int64_t need = (int64_t)h->sym.n * nrhs;
  if (need <= h->x_cap) return SPB_OK;
  for (double** p : {&h->dX, &h->dZ, &h->dB, &h->dR, &h->dD, &h->dXo}) {
    if (*p) {
      auto it = std::find(h->allocs.begin(), h->allocs.end(), (void*)*p);
      if (it != h->allocs.end()) h->allocs.erase(it);
      cudaStreamSynchronize(h->stream);
      cudaFreeAsync(*p, h->own_stream);
      h->device_bytes -= h->x_cap * (int64_t)sizeof(double);
      *p = nullptr;
    }
  }
  h->x_cap = 0;
  SPB_CK(h, dalloc(h, &h->dX, need));
  SPB_CK(h, dalloc(h, &h->dZ, need));
  SPB_CK(h, dalloc(h, &h->dB, need));
  if (h->fp32) {
    SPB_CK(h, dalloc(h, &h->dR, need));
    SPB_CK(h, dalloc(h, &h->dD, need));
    SPB_CK(h, dalloc(h, &h->dXo, need));
  }
  h->x_cap = need;
  SPB_CK(h, cudaStreamSynchronize(h->own_stream));  // allocations usable from any stream
  return SPB_OK;
}

// Diagonal super-block inverses of the current factor, computed by the first solve
// after a factorization.
void ensure_inverses(spb_handle* h) {
  if (!h->inv_stale) return;
  const spb::Plan& P = h->plan;
  const int count = (int)P.inv_items.size();
  spb::dev::launch_sb_inverse(h->stream, h->ldl ? (const void*)h->dW : h->dL, h->dInv, h->fp32, h->dmeta,
                              h->dinvitems, count, P.solve_sb);
  if (h->ldl) spb::dev::launch_sb_inverse(h->stream, h->dL, h->dInvB, false, h->dmeta, h->dinvitems, count, P.solve_sb);
  h->inv_stale = false;
}

// Forward and backward persistent sweeps on the permuted right-hand sides X (n x nrhs,
// ld n; the solution replaces them), with Z (same shape) between the sweeps and the
// counters in sync; 64 right-hand sides per pass.  prof: record the per-pass events.
void enqueue_sweeps(spb_handle* h, double* X, double* Z, int32_t* sync, int nrhs, bool prof) {
  const spb::Plan& P = h->plan;
  const int ns = P.nsuper;
  for (int c0 = 0; c0 < nrhs; c0 += 64) {
    // counters must start at zero
    cudaMemsetAsync(sync, 0, sizeof(int32_t) * spb::solve_sync_ints(P), h->stream);
    spb::dev::PSolveArgs a{};
    // LDL^T: the forward sweep solves with L D (diagonal D), the backward one with unit L
    a.L = h->ldl ? (void*)h->dW : h->dL;
    a.Inv = h->dInv;
    a.fp32 = h->fp32;
    a.meta = h->dmeta;
    a.rows = h->drows;
    a.supmember = h->dsupm;
    a.sparent = h->dsparent;
    a.row_group = h->drowgrp;
    a.groups = h->dgroups;
    a.X = X + (int64_t)c0 * h->sym.n;
    a.Z = Z + (int64_t)c0 * h->sym.n;
    a.ldx = h->sym.n;
    a.nrhs = std::min(64, nrhs - c0);
    a.expected = h->dexpected;
    a.tiny = h->dtiny;
    a.arrived = sync + 2;
    a.status = h->dstatus;
    a.spin_limit = h->wait_limit;
    a.sb = P.solve_sb;
    a.tpt = P.solve_tpt;
    const size_t e0 = 4 * (size_t)(c0 / 64);
    a.tasks = h->dfwd;
    a.ntasks = (int)P.fwd_tasks.size();
    a.counter = sync;
    a.blkdone = sync + 2 + ns;
    a.upd = sync + 2 + 3 * (size_t)ns;
    a.trace = prof ? h->dtrace : nullptr;
    const size_t pass_bytes = sizeof(double) * (size_t)h->sym.n * a.nrhs;
    if (prof) cudaEventRecord(h->events[e0], h->stream);
    cudaMemsetAsync(a.Z, 0, pass_bytes, h->stream);  // DI tasks of wide supernodes add into Z
    spb::dev::launch_solve_persistent(h->stream, a, true);
    if (prof) cudaEventRecord(h->events[e0 + 1], h->stream);
    a.L = h->dL;
    a.Inv = h->ldl ? h->dInvB : h->dInv;
    a.tasks = h->dbwd;
    a.ntasks = (int)P.bwd_tasks.size();
    a.counter = sync + 1;
    a.blkdone = sync + 2 + 2 * ns;
    a.upd = sync + 2 + 3 * (size_t)ns + P.nsb_total;
    a.trace = prof && h->dtrace ? h->dtrace + 4 * P.fwd_tasks.size() : nullptr;
    if (prof) cudaEventRecord(h->events[e0 + 2], h->stream);
    cudaMemsetAsync(a.X, 0, pass_bytes, h->stream);  // the backward DI tasks add into X
    spb::dev::launch_solve_persistent(h->stream, a, false);
    if (prof) cudaEventRecord(h->events[e0 + 3], h->stream);
  }
}

// Both sweeps on the handle's workspace h->dX (n x nrhs, ld n), inverses first if stale.
void enqueue_solve(spb_handle* h, int nrhs) {
  // per-pass events of a profiled solve (every caller, the refinement loop included)
  const bool prof = h->profiling && ensure_events(h, 4 * (size_t)((nrhs + 63) / 64) + 2) == cudaSuccess;
  const size_t ie = 4 * (size_t)((nrhs + 63) / 64);
  const bool inv = h->inv_stale;
  if (prof) cudaEventRecord(h->events[ie], h->stream);
  ensure_inverses(h);
  if (prof) cudaEventRecord(h->events[ie + 1], h->stream);
  h->prof_inverse = prof && inv;
  enqueue_sweeps(h, h->dX, h->dZ, h->dsync, nrhs, prof);
}

// Per-sweep device times of the last profiled solve.
int collect_solve_profile(spb_handle* h, int nrhs) {
  if (!h->profiling) return SPB_OK;
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  clear_kinds(h, SPB_KIND_SOLVE_FORWARD, SPB_KIND_SOLVE_BACKWARD);
  h->prof.ms[SPB_KIND_SOLVE_INVERSE] = 0.0;
  h->prof.launches[SPB_KIND_SOLVE_INVERSE] = 0;
  h->prof.flops[SPB_KIND_SOLVE_INVERSE] = 0.0;
  if (h->prof_inverse) {  // the first solve after a factorization computed the inverses
    const size_t ie = 4 * (size_t)((nrhs + 63) / 64);
    float ms = 0.f;
    SPB_CK(h, cudaEventElapsedTime(&ms, h->events[ie], h->events[ie + 1]));
    h->prof.ms[SPB_KIND_SOLVE_INVERSE] = ms;
    h->prof.launches[SPB_KIND_SOLVE_INVERSE] = h->ldl ? 2 : 1;
  }
  for (int c0 = 0, i = 0; c0 < nrhs; c0 += 64, ++i) {
    float f = 0.f, b = 0.f;
    SPB_CK(h, cudaEventElapsedTime(&f, h->events[4 * i], h->events[4 * i + 1]));
    SPB_CK(h, cudaEventElapsedTime(&b, h->events[4 * i + 2], h->events[4 * i + 3]));
    const double rhs_bytes = 16.0 * h->sym.n * std::min(64, nrhs - c0);  // X read and written once
    h->prof.ms[SPB_KIND_SOLVE_FORWARD] += f;
    h->prof.ms[SPB_KIND_SOLVE_BACKWARD] += b;
    h->prof.bytes[SPB_KIND_SOLVE_FORWARD] += h->plan.solve_sweep_bytes + rhs_bytes;
    h->prof.bytes[SPB_KIND_SOLVE_BACKWARD] += h->plan.solve_sweep_bytes + rhs_bytes;
    h->prof.launches[SPB_KIND_SOLVE_FORWARD] += 1;
    h->prof.launches[SPB_KIND_SOLVE_BACKWARD] += 1;
  }
  return SPB_OK;
}

// Status word after a solve: device waits are bounded, report their expiry.
int check_solve_status(spb_handle* h) {
  Status st;
  SPB_CK(h, cudaMemcpyAsync(&st, h->dstatus, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  if (st.code == 3) {
    // the context is intact: clear the word so the next solve can run
    SPB_CK(h, cudaMemsetAsync(h->dstatus, 0, sizeof(Status), h->stream));
    SPB_CK(h, cudaStreamSynchronize(h->stream));
    char msg[96];
    snprintf(msg, sizeof msg, "solve: a device wait expired (supernode %d)", st.supernode + 1);
    return fail(h, SPB_ERR_TIMEOUT, msg);
  }
  if (st.code != 0 && st.code != 1) return fail(h, SPB_ERR_STRUCTURE, "solve: device status error");
  return SPB_OK;
}

// Solve with the factor as it is: b (ld ldb) -> x (ld ldx), through the permuted workspace.
void plain_solve(spb_handle* h, const double* b, int64_t ldb, double* x, int64_t ldx, int nrhs) {
  const int n = h->sym.n;
  spb::dev::launch_permute_in(h->stream, h->dX, n, b, ldb, h->dinvp0, n, nrhs);
  enqueue_solve(h, nrhs);
  spb::dev::launch_permute_out(h->stream, x, ldx, h->dX, n, h->dinvp0, n, nrhs);
}

// Precision form: solve with the FP32 factor, then refine in FP64 until the
// backward error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) of every
// right-hand side is at most ir_tolerance.  b and x are in the original order.
int ir_solve(spb_handle* h, const double* d_b, int64_t ldb, double* d_x, int64_t ldx, int nrhs) {
  const int n = h->sym.n;
  const double tol = h->opt.ir_tolerance > 0 ? h->opt.ir_tolerance : 1e-12;
  const int maxit = h->opt.ir_max_iter > 0 ? h->opt.ir_max_iter : 30;
  int iters_all = 0;
  double eta_all = 0.0;
  for (int c0 = 0; c0 < nrhs; c0 += 64) {
    const int nr = std::min(64, nrhs - c0);
    const double* b = d_b + (int64_t)c0 * ldb;
    double* x = d_x + (int64_t)c0 * ldx;
    plain_solve(h, b, ldb, x, ldx, nr);
    const int nseg = num_segments(h);
    double* anorm = h->d_norms + 1;
    double* bmax = anorm + nseg;
    double* xmax = bmax + (size_t)nseg * 64;
    double* rmax = xmax + (size_t)nseg * 64;
    SPB_CK(h, cudaMemsetAsync(bmax, 0, sizeof(double) * 64 * (size_t)nseg, h->stream));
    spb::dev::launch_segmax(h->stream, b, n, nr, ldb, h->d_rowseg, bmax);
    double eta = 0.0, eta_prev = 1e300;
    int it = 0;
    for (;;) {
      spb::dev::launch_residual(h->stream, h->d_rowptr, h->d_col, h->d_val, x, b, h->dR, n, nr, ldx);
      SPB_CK(h, cudaMemsetAsync(xmax, 0, sizeof(double) * 128 * (size_t)nseg, h->stream));
      SPB_CK(h, cudaMemsetAsync(h->d_norms, 0, sizeof(double), h->stream));
      spb::dev::launch_segmax(h->stream, x, n, nr, ldx, h->d_rowseg, xmax);
      spb::dev::launch_segmax(h->stream, h->dR, n, nr, ldx, h->d_rowseg, rmax);
      spb::dev::launch_eta(h->stream, anorm, bmax, xmax, rmax, nseg, nr, h->d_norms);
      SPB_CK(h, cudaMemcpyAsync(&eta, h->d_norms, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      int rc = check_solve_status(h);  // synchronizes
      if (rc) return rc;
      if (eta <= tol) break;
      if (it >= maxit || (it >= 4 && eta > 0.9 * eta_prev)) {
        h->ir_iterations = std::max(iters_all, it);
        h->backward_error = std::max(eta_all, eta);
        char msg[128];
        snprintf(msg, sizeof msg, "refinement stopped at backward error %.3e after %d steps (target %.1e)", eta, it,
                 tol);
        return fail(h, SPB_ERR_NOT_CONVERGED, msg);
      }
      eta_prev = eta;
      plain_solve(h, h->dR, ldx, h->dD, ldx, nr);
      spb::dev::launch_axpy(h->stream, x, h->dD, n, nr, ldx);
      ++it;
    }
    iters_all = std::max(iters_all, it);
    eta_all = std::max(eta_all, eta);
  }
  h->ir_iterations = iters_all;
  h->backward_error = eta_all;
  return SPB_OK;
}

}  // namespace

extern "C" {

void spb_default_options(spb_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->ordering = SPB_ORDERING_MMD;
  o->nrelax0 = 8;
  o->nrelax1 = 32;
  o->nrelax2 = 64;
  o->max_snode = 0;
  o->zrelax0 = 0.8;
  o->zrelax1 = 0.1;
  o->zrelax2 = 0.05;
  o->user_perm = nullptr;
  o->device = 0;
  o->precision = SPB_PRECISION_FP64;
  o->ir_tolerance = 1e-12;
  o->ir_max_iter = 30;
  o->verbose = 0;
  o->decomposition = SPB_DECOMPOSITION_LL;
  o->fp32_engine = 3;
  o->factor_schedule = SPB_FACTOR_AUTO;
}

int spb_create(const spb_options* opt, spb_handle** out) {
  if (!out) return SPB_ERR_INVALID;
  *out = nullptr;
  spb_handle* h = new (std::nothrow) spb_handle();
  if (!h) return SPB_ERR_OOM;
  if (opt) h->opt = *opt;
  else spb_default_options(&h->opt);
  if (h->opt.ordering < 0 || h->opt.ordering > 4 || h->opt.precision < 0 || h->opt.precision > 1 ||
      h->opt.fp32_engine < 0 || h->opt.fp32_engine > 3 || h->opt.decomposition < 0 || h->opt.decomposition > 1 ||
      h->opt.plan_outer_nb < 0 || h->opt.plan_outer_nb > 4096 || h->opt.plan_outer_nb % 64 ||
      h->opt.factor_schedule < SPB_FACTOR_AUTO || h->opt.factor_schedule > SPB_FACTOR_PERSISTENT ||
      (h->opt.decomposition == SPB_DECOMPOSITION_LDL && h->opt.precision != SPB_PRECISION_FP64)) {
    delete h;
    return SPB_ERR_INVALID;
  }
  h->device = h->opt.device;
  if (h->device < 0) {  // host-only handle: symbolic analysis and introspection, no CUDA
    *out = h;
    return SPB_OK;
  }
  cudaError_t e = cudaSetDevice(h->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->side_stream, cudaStreamNonBlocking);
  h->stream = h->own_stream;
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
    return e == cudaErrorMemoryAllocation ? SPB_ERR_OOM : SPB_ERR_CUDA;
  }
  {
    // kernel attributes are per device; handles may be created from several threads
    static std::mutex mu;
    static bool done[256] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (h->device < 256 && !done[h->device]) {
      spb::dev::init_kernel_attributes();
      done[h->device] = true;
    } else if (h->device >= 256) {
      spb::dev::init_kernel_attributes();
    }
  }
  *out = h;
  return SPB_OK;
}

void spb_destroy(spb_handle* h) {
  if (!h) return;
  if (h->device < 0) {
    delete h;
    return;
  }
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  release_device(h);
  for (cudaEvent_t e : h->events) cudaEventDestroy(e);
  for (cudaEvent_t e : h->lane_events) cudaEventDestroy(e);
  if (h->side_stream) cudaStreamDestroy(h->side_stream);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
}

const char* spb_last_error(const spb_handle* h) { return h ? h->err.c_str() : "null handle"; }

}  // extern "C"

namespace {

spb::RelaxParams relax_of(const spb_options& o) {
  spb::RelaxParams rp;
  rp.nrelax0 = o.nrelax0;
  rp.nrelax1 = o.nrelax1;
  rp.nrelax2 = o.nrelax2;
  rp.maxSize = o.max_snode;
  rp.zrelax0 = o.zrelax0;
  rp.zrelax1 = o.zrelax1;
  rp.zrelax2 = o.zrelax2;
  if (rp.maxSize > 0) {  // RelaxationParameters::SetMaxSize (Types.hpp:63-70)
    rp.nrelax0 = std::min(rp.nrelax0, rp.maxSize);
    rp.nrelax1 = std::min(rp.nrelax1, rp.maxSize);
    rp.nrelax2 = std::min(rp.nrelax2, rp.maxSize);
  }
  return rp;
}

spb::PlanParams plan_params_of(const spb_options& o) {
  spb::PlanParams pp;
  if (o.device >= 0) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o.device) == cudaSuccess && sms > 0) pp.sms = sms;
  }
  if (o.plan_small_max_w > 0) pp.small_max_w = o.plan_small_max_w;
  if (o.plan_big_tile_rows > 0) pp.big_tile_rows = o.plan_big_tile_rows;
  if (o.plan_outer_nb > 0) pp.outer_nb = o.plan_outer_nb;
  if (o.plan_solve_chunk > 0) pp.solve_sb = o.plan_solve_chunk;
  if (o.plan_solve_tiles > 0) pp.solve_tpt = o.plan_solve_tiles;
  pp.factor_dag = persistent_schedule(o);
  pp.fp32 = o.precision == SPB_PRECISION_FP32_IR;
  return pp;
}

// Map index of every supernode that owns 128 x 128 tiles (-1 for the others); returns the count.
int tile_map_index(const spb::Plan& P, std::vector<int32_t>& of) {
  of.assign(P.nsuper, -1);
  int n = 0;
  for (const spb::Step& st : P.steps) {
    if (st.kind != spb::StepKind::Gemm || st.tile != 128) continue;
    for (int i = st.begin; i < st.begin + st.count; ++i) {
      const int s = P.tile_items[i].s;
      if (of[s] < 0) of[s] = n++;
    }
  }
  return n;
}

// Floats of the split copies (hi and lo rows of every panel with 128 x 128 tiles), the
// offset of each supernode's copy (-1: none) in `off`.
int64_t split_layout(const spb::Plan& P, const std::vector<int32_t>& of, std::vector<int64_t>& off) {
  off.assign(P.nsuper, -1);
  int64_t t = 0;
  for (int s = 0; s < P.nsuper; ++s) {
    if (of[s] < 0) continue;
    const spb::SnMeta& m = P.meta[s];
    off[s] = t;
    t += (2 * (int64_t)m.h * ((m.w + 3) & ~3) + 31) / 32 * 32;  // 128-byte aligned copies
  }
  return t;
}

// Split copies of the FP32 panels read by the TMA-fed tcgen05 tiles, and their 3-D tiled
// tensor maps: columns inner (extent w, pitch round_up(w, 4)), rows (extent h), then
// {hi, lo}; 32 x 128 x 2 boxes, 128-byte swizzle, zero outside the panel.  Checks the
// tile shape that engine relies on (a K range of whole 32-column chunks, or one ending at
// the panel's last column).
int build_tile_maps(spb_handle* h) {
  const spb::Plan& P = h->plan;
  std::vector<int32_t> of;
  const int nmaps = tile_map_index(P, of);
  for (const spb::Step& st : P.steps) {
    if (st.kind != spb::StepKind::Gemm || st.tile != 128) continue;
    for (int i = st.begin; i < st.begin + st.count; ++i) {
      const spb::TileItem& t = P.tile_items[i];
      if (!(t.kn % 32 == 0 || t.k0 + t.kn == P.meta[t.s].w) || t.k0 % 4)
        return fail(h, SPB_ERR_STRUCTURE, "plan: a 128 x 128 tile does not fit the TMA-fed engine");
    }
  }
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return fail(h, SPB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  std::vector<int64_t> off;
  const int64_t floats = split_layout(P, of, off);
  SPB_CK(h, dalloc(h, &h->dsplit, (size_t)floats));
  SPB_CK(h, dalloc(h, &h->dsplit_off, off.size()));
  SPB_CK(h, dalloc(h, &h->dtmaps, (size_t)std::max(nmaps, 1)));
  SPB_CK(h, dalloc(h, &h->dtmap_of, of.size()));
  std::vector<CUtensorMap> maps(std::max(nmaps, 1));
  for (int s = 0; s < P.nsuper; ++s) {
    if (of[s] < 0) continue;
    const spb::SnMeta& m = P.meta[s];
    const cuuint64_t pitch = (cuuint64_t)((m.w + 3) & ~3);
    cuuint64_t dims[3] = {(cuuint64_t)m.w, (cuuint64_t)m.h, 2};
    cuuint64_t strides[2] = {pitch * sizeof(float), pitch * (cuuint64_t)m.h * sizeof(float)};
    cuuint32_t box[3] = {32, 128, 2}, es[3] = {1, 1, 1};
    const CUresult r = encode(&maps[of[s]], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, h->dsplit + off[s], dims, strides,
                              box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(h, SPB_ERR_CUDA, "cuTensorMapEncodeTiled failed for a panel");
  }
  SPB_CK(h, cudaStreamSynchronize(h->own_stream));
  SPB_CK(h, cudaMemcpyAsync(h->dtmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice,
                            h->stream));
  SPB_CK(h, cudaMemcpyAsync(h->dtmap_of, of.data(), of.size() * 4, cudaMemcpyHostToDevice, h->stream));
  SPB_CK(h, cudaMemcpyAsync(h->dsplit_off, off.data(), off.size() * 8, cudaMemcpyHostToDevice, h->stream));
  SPB_CK(h, cudaStreamSynchronize(h->stream));  // the host copies go out of scope
  return SPB_OK;
}

int begin_symbolic(spb_handle* h, int32_t n, const int64_t* colptr, const int32_t* rowind) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (n <= 0 || !colptr || !rowind) return fail(h, SPB_ERR_INVALID, "symbolic: empty matrix or null pointer");
  if (h->device >= 0) {
    SPB_CK(h, cudaSetDevice(h->device));
    release_device(h);
  }
  h->have_symbolic = h->have_values = h->factored = h->have_solution = false;
  h->cells_built = false;
  h->nnz_a = colptr[n] - 1;
  h->seg_off.clear();
  h->colptr.assign(colptr, colptr + n + 1);
  h->rowind.assign(rowind, rowind + h->nnz_a);
  return SPB_OK;
}

// Everything after the symbolic analysis: device plan, assembly map and the
// handle's device buffers.  h->sym must hold the (possibly merged) analysis.
int install_device(spb_handle* h);

// Device bytes install_device + a solve of nrhs right-hand sides allocate
// (the same list of buffers, sizes as requested from cudaMalloc).  The plan depends on
// the precision (tile shapes, task graph), so a prediction for the other precision plans
// the analysis for it (once per handle and precision).
int64_t predict_bytes(const spb_handle* h, bool fp32, int nrhs) {
  spb_options o = h->opt;
  o.precision = fp32 ? SPB_PRECISION_FP32_IR : SPB_PRECISION_FP64;
  const spb::PlanParams want = plan_params_of(o);
  const spb::Plan* plan = &h->plan;
  if (!(want == plan_params_of(h->opt))) {
    std::lock_guard<std::mutex> lock(h->pred_mu);
    std::unique_ptr<spb::Plan>& c = h->pred_plan[fp32 ? 1 : 0];
    if (!c || !(h->pred_prm[fp32 ? 1 : 0] == want)) {
      c = std::make_unique<spb::Plan>(spb::build_plan(h->sym, want));
      h->pred_prm[fp32 ? 1 : 0] = want;
    }
    plan = c.get();
  }
  const spb::Plan& P = *plan;
  const int64_t n = h->sym.n, ns = P.nsuper;
  auto b = [](int64_t count, size_t size) { return std::max<int64_t>(count, 1) * (int64_t)size; };
  int64_t t = b(P.arena_elems, fp32 ? sizeof(float) : sizeof(double));
  if (o.decomposition == SPB_DECOMPOSITION_LDL) t += b(P.arena_elems, sizeof(double));
  t += b(P.meta.size(), sizeof(spb::SnMeta)) + b(P.rows.size(), 4) + b(P.supmember0.size(), 4);
  t += b(P.row_group.size(), 4) + b(P.groups.size(), sizeof(spb::RelGroup)) + b(P.rel.size(), 4);
  t += b(h->amap.size(), 8) + b(h->nnz_a, 8) + b(P.small_items.size(), 4);
  t += b(P.panel_items.size(), sizeof(spb::PanelItem));
  t += b((int64_t)std::max(1, P.max_diag_slots) * (int64_t)spb::dev::kDiagSlotDoubles, 8);
  t += b(P.tile_items.size(), sizeof(spb::TileItem)) + b(n, 4) + b(ns, 4);
  t += b(P.fwd_tasks.size(), sizeof(spb::SolveTask)) + b(P.bwd_tasks.size(), sizeof(spb::SolveTask));
  t += b(P.fwd_pending.size(), 4) + b(P.tiny.size(), 4) + b(P.sparent.size(), 4) +
       b((int64_t)spb::solve_sync_ints(P), 4);
  t += b(P.inv_elems, fp32 ? sizeof(float) : sizeof(double)) + b(P.inv_items.size(), sizeof(spb::InvItem));
  t += b(P.ftasks.size(), sizeof(spb::FTask)) + b(P.fwaits.size(), sizeof(spb::FWait)) + b(P.fsigs.size(), 4) +
       b(P.nfctr + 1, 4);
  if (o.decomposition == SPB_DECOMPOSITION_LDL) t += b(P.inv_elems, sizeof(double));
  t += b(1, sizeof(Status));
  if (fp32) {
    int64_t offdiag = 0;
    for (int64_t c = 1; c <= n; ++c)
      for (int64_t p = h->colptr[c - 1]; p < h->colptr[c]; ++p) offdiag += h->rowind[p - 1] != c;
    const int64_t nnz_full = h->nnz_a + offdiag;
    t += b(n + 1, 8) + b(nnz_full, 4) + b(nnz_full, 8) + b(nnz_full, 8);
    t += b(1 + (int64_t)num_segments(h) * (1 + 3 * 64), 8);
    if (!h->seg_off.empty()) t += b(n, 4);
  }
  if (fp32 && o.fp32_engine == 3) {
    std::vector<int32_t> of;
    std::vector<int64_t> off;
    const int nmaps = tile_map_index(P, of);
    t += b(split_layout(P, of, off), sizeof(float)) + b(ns, 8) + b(nmaps, sizeof(CUtensorMap)) + b(ns, 4);
  }
  if (nrhs > 0) t += (fp32 ? 6 : 3) * b(n * nrhs, 8);
  return t;
}

int install_symbolic(spb_handle* h, int32_t n, const int64_t* colptr, const int32_t* rowind) {
  try {
    h->plan = spb::build_plan(h->sym, plan_params_of(h->opt));
    h->amap = spb::build_assembly_map(h->sym, h->plan, colptr, rowind);
  } catch (const std::bad_alloc&) {
    return fail(h, SPB_ERR_OOM, "symbolic: host allocation failed");
  } catch (const std::exception& e) {
    return fail(h, SPB_ERR_STRUCTURE, e.what());
  }
  return install_device(h);
}

// Device buffers of an analysed handle (h->sym, h->plan, h->amap, h->colptr and
// h->rowind set); a host-only handle just records that the analysis is done.
int install_device(spb_handle* h) {
  {  // a new analysis: earlier predictions' plans are stale
    std::lock_guard<std::mutex> lock(h->pred_mu);
    h->pred_plan[0].reset();
    h->pred_plan[1].reset();
  }
  if (h->device < 0) {
    h->have_symbolic = true;
    return SPB_OK;
  }
  const int32_t n = h->sym.n;
  const int64_t* colptr = h->colptr.data();
  const int32_t* rowind = h->rowind.data();
  const std::vector<int64_t>& amap = h->amap;
  const spb::Plan& P = h->plan;
  std::vector<int32_t> lsn, invp0(n);
  h->level_off.assign(P.nlevels + 1, 0);
  for (int l = 0; l < P.nlevels; ++l) {
    h->level_off[l] = (int32_t)lsn.size();
    lsn.insert(lsn.end(), P.level_sn[l].begin(), P.level_sn[l].end());
  }
  h->level_off[P.nlevels] = (int32_t)lsn.size();
  for (int i = 0; i < n; ++i) invp0[i] = h->sym.invp[i] - 1;

  h->fp32 = h->opt.precision == SPB_PRECISION_FP32_IR;
  h->ldl = h->opt.decomposition == SPB_DECOMPOSITION_LDL;
  h->elem = h->fp32 ? sizeof(float) : sizeof(double);
  {
    unsigned char* arena = nullptr;
    SPB_CK(h, dalloc(h, &arena, (size_t)P.arena_elems * h->elem));
    h->dL = arena;
  }
  if (h->ldl) SPB_CK(h, dalloc(h, &h->dW, (size_t)P.arena_elems));
  SPB_CK(h, dalloc(h, &h->dmeta, P.meta.size()));
  SPB_CK(h, dalloc(h, &h->drows, P.rows.size()));
  SPB_CK(h, dalloc(h, &h->dsupm, P.supmember0.size()));
  SPB_CK(h, dalloc(h, &h->drowgrp, P.row_group.size()));
  SPB_CK(h, dalloc(h, &h->dgroups, P.groups.size()));
  SPB_CK(h, dalloc(h, &h->drel, P.rel.size()));
  SPB_CK(h, dalloc(h, &h->damap, amap.size()));
  SPB_CK(h, dalloc(h, &h->dA, (size_t)h->nnz_a));
  SPB_CK(h, dalloc(h, &h->dsmall, P.small_items.size()));
  SPB_CK(h, dalloc(h, &h->dpanel, P.panel_items.size()));
  SPB_CK(h, dalloc(h, &h->dwinv, (size_t)std::max(1, P.max_diag_slots) * spb::dev::kDiagSlotDoubles));
  SPB_CK(h, dalloc(h, &h->dtiles, P.tile_items.size()));
  SPB_CK(h, dalloc(h, &h->dinvp0, invp0.size()));
  SPB_CK(h, dalloc(h, &h->dlevel_sn, lsn.size()));
  SPB_CK(h, dalloc(h, &h->dfwd, P.fwd_tasks.size()));
  SPB_CK(h, dalloc(h, &h->dbwd, P.bwd_tasks.size()));
  SPB_CK(h, dalloc(h, &h->dexpected, P.fwd_pending.size()));
  SPB_CK(h, dalloc(h, &h->dtiny, P.tiny.size()));
  SPB_CK(h, dalloc(h, &h->dsparent, P.sparent.size()));
  SPB_CK(h, dalloc(h, &h->dsync, spb::solve_sync_ints(P)));
  {
    unsigned char* inv = nullptr;
    SPB_CK(h, dalloc(h, &inv, (size_t)P.inv_elems * h->elem));
    h->dInv = inv;
  }
  SPB_CK(h, dalloc(h, &h->dinvitems, P.inv_items.size()));
  SPB_CK(h, dalloc(h, &h->dftasks, P.ftasks.size()));
  SPB_CK(h, dalloc(h, &h->dfwaits, P.fwaits.size()));
  SPB_CK(h, dalloc(h, &h->dfsigs, P.fsigs.size()));
  SPB_CK(h, dalloc(h, &h->dfctr, (size_t)P.nfctr + 1));
  if (h->ldl) {
    double* invb = nullptr;
    SPB_CK(h, dalloc(h, &invb, (size_t)P.inv_elems));
    h->dInvB = invb;
  } else {
    h->dInvB = h->dInv;
  }
  h->inv_stale = true;
  SPB_CK(h, dalloc(h, &h->dstatus, 1));
  SPB_CK(h, cudaStreamSynchronize(h->own_stream));  // allocations ready before h->stream uses them
  auto up = [&](void* d, const void* s, size_t bytes) {
    return bytes ? cudaMemcpyAsync(d, s, bytes, cudaMemcpyHostToDevice, h->stream) : cudaSuccess;
  };
  SPB_CK(h, up(h->dmeta, P.meta.data(), P.meta.size() * sizeof(spb::SnMeta)));
  SPB_CK(h, up(h->drows, P.rows.data(), P.rows.size() * 4));
  SPB_CK(h, up(h->dsupm, P.supmember0.data(), P.supmember0.size() * 4));
  SPB_CK(h, up(h->drowgrp, P.row_group.data(), P.row_group.size() * 4));
  SPB_CK(h, up(h->dgroups, P.groups.data(), P.groups.size() * sizeof(spb::RelGroup)));
  SPB_CK(h, up(h->drel, P.rel.data(), P.rel.size() * 4));
  SPB_CK(h, up(h->damap, amap.data(), amap.size() * 8));
  SPB_CK(h, up(h->dsmall, P.small_items.data(), P.small_items.size() * 4));
  SPB_CK(h, up(h->dpanel, P.panel_items.data(), P.panel_items.size() * sizeof(spb::PanelItem)));
  SPB_CK(h, up(h->dtiles, P.tile_items.data(), P.tile_items.size() * sizeof(spb::TileItem)));
  SPB_CK(h, up(h->dinvp0, invp0.data(), invp0.size() * 4));
  SPB_CK(h, up(h->dlevel_sn, lsn.data(), lsn.size() * 4));
  SPB_CK(h, up(h->dfwd, P.fwd_tasks.data(), P.fwd_tasks.size() * sizeof(spb::SolveTask)));
  SPB_CK(h, up(h->dbwd, P.bwd_tasks.data(), P.bwd_tasks.size() * sizeof(spb::SolveTask)));
  SPB_CK(h, up(h->dexpected, P.fwd_pending.data(), P.fwd_pending.size() * 4));
  SPB_CK(h, up(h->dtiny, P.tiny.data(), P.tiny.size() * 4));
  SPB_CK(h, up(h->dsparent, P.sparent.data(), P.sparent.size() * 4));
  SPB_CK(h, up(h->dinvitems, P.inv_items.data(), P.inv_items.size() * sizeof(spb::InvItem)));
  SPB_CK(h, up(h->dftasks, P.ftasks.data(), P.ftasks.size() * sizeof(spb::FTask)));
  SPB_CK(h, up(h->dfwaits, P.fwaits.data(), P.fwaits.size() * sizeof(spb::FWait)));
  SPB_CK(h, up(h->dfsigs, P.fsigs.data(), P.fsigs.size() * 4));
  h->trace_fresh = false;
  SPB_CK(h, cudaMemsetAsync(h->dstatus, 0, sizeof(Status), h->stream));
  if (h->fp32 && h->opt.fp32_engine == 3) {
    const int rc = build_tile_maps(h);
    if (rc != SPB_OK) return rc;
  }
  if (h->fp32) {
    // full symmetric CSR of A in the original ordering; csr_src maps each entry to its input value
    std::vector<int64_t>& rp = h->csr_rowptr;
    rp.assign(n + 1, 0);
    for (int c = 1; c <= n; ++c)
      for (int64_t p = colptr[c - 1]; p < colptr[c]; ++p) {
        int r = rowind[p - 1];
        rp[r]++;
        if (r != c) rp[c]++;
      }
    for (int i = 0; i < n; ++i) rp[i + 1] += rp[i];
    h->csr_col.assign(rp[n], 0);
    h->csr_src.assign(rp[n], 0);
    std::vector<int64_t> fill(rp.begin(), rp.end() - 1);
    for (int c = 1; c <= n; ++c)
      for (int64_t p = colptr[c - 1]; p < colptr[c]; ++p) {
        int r = rowind[p - 1];
        int64_t k = fill[r - 1]++;
        h->csr_col[k] = c - 1;
        h->csr_src[k] = p - 1;
        if (r != c) {
          k = fill[c - 1]++;
          h->csr_col[k] = r - 1;
          h->csr_src[k] = p - 1;
        }
      }
    SPB_CK(h, dalloc(h, &h->d_rowptr, rp.size()));
    SPB_CK(h, dalloc(h, &h->d_col, h->csr_col.size()));
    SPB_CK(h, dalloc(h, &h->d_csrsrc, h->csr_src.size()));
    SPB_CK(h, dalloc(h, &h->d_val, h->csr_col.size()));
    SPB_CK(h, dalloc(h, &h->d_norms, 1 + (size_t)num_segments(h) * (1 + 3 * 64)));
    if (!h->seg_off.empty()) {
      std::vector<int32_t> rowseg(n);
      for (size_t k = 0; k + 1 < h->seg_off.size(); ++k)
        for (int32_t i = h->seg_off[k]; i < h->seg_off[k + 1]; ++i) rowseg[i] = (int32_t)k;
      SPB_CK(h, dalloc(h, &h->d_rowseg, rowseg.size()));
      SPB_CK(h, cudaStreamSynchronize(h->own_stream));
      SPB_CK(h, cudaMemcpyAsync(h->d_rowseg, rowseg.data(), rowseg.size() * 4, cudaMemcpyHostToDevice, h->stream));
    }
    SPB_CK(h, cudaStreamSynchronize(h->own_stream));
    SPB_CK(h, up(h->d_rowptr, rp.data(), rp.size() * 8));
    SPB_CK(h, up(h->d_col, h->csr_col.data(), h->csr_col.size() * 4));
    SPB_CK(h, up(h->d_csrsrc, h->csr_src.data(), h->csr_src.size() * 8));
  }
  SPB_CK(h, cudaStreamSynchronize(h->own_stream));
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  h->have_symbolic = true;
  return SPB_OK;
}

}  // namespace

extern "C" {

int spb_symbolic(spb_handle* h, int32_t n, const int64_t* colptr, const int32_t* rowind) {
  int rc = begin_symbolic(h, n, colptr, rowind);
  if (rc) return rc;
  try {
    h->sym = spb::symbolic_factorization(n, colptr, rowind, (spb::OrderingKind)h->opt.ordering, relax_of(h->opt),
                                         h->opt.user_perm);
  } catch (const std::invalid_argument& e) {
    return fail(h, SPB_ERR_INVALID, e.what());
  } catch (const std::bad_alloc&) {
    return fail(h, SPB_ERR_OOM, "symbolic: host allocation failed");
  } catch (const std::exception& e) {
    return fail(h, SPB_ERR_STRUCTURE, e.what());
  }
  return install_symbolic(h, n, colptr, rowind);
}

int spb_symbolic_from(spb_handle* h, const spb_handle* src) {
  if (check_handle(h) || !src) return SPB_ERR_INVALID;
  if (h == src) return fail(h, SPB_ERR_INVALID, "symbolic_from: source is the handle itself");
  if (!src->have_symbolic) return fail(h, SPB_ERR_STATE, "symbolic_from: source has no symbolic analysis");
  if (h->opt.ordering != src->opt.ordering || h->opt.nrelax0 != src->opt.nrelax0 ||
      h->opt.nrelax1 != src->opt.nrelax1 || h->opt.nrelax2 != src->opt.nrelax2 ||
      h->opt.max_snode != src->opt.max_snode || h->opt.zrelax0 != src->opt.zrelax0 ||
      h->opt.zrelax1 != src->opt.zrelax1 || h->opt.zrelax2 != src->opt.zrelax2)
    return fail(h, SPB_ERR_INVALID, "symbolic_from: ordering / relaxation options differ from the source's");
  if (h->device >= 0) {
    SPB_CK(h, cudaSetDevice(h->device));
    release_device(h);
  }
  h->have_symbolic = h->have_values = h->factored = h->have_solution = false;
  h->cells_built = false;
  try {
    h->sym = src->sym;
    h->seg_off = src->seg_off;
    h->nnz_a = src->nnz_a;
    h->colptr = src->colptr;
    h->rowind = src->rowind;
    if (plan_params_of(h->opt) == plan_params_of(src->opt)) {  // same tunables: the same plan
      h->plan = src->plan;
      h->amap = src->amap;
    } else {
      h->plan = spb::build_plan(h->sym, plan_params_of(h->opt));
      h->amap = spb::build_assembly_map(h->sym, h->plan, h->colptr.data(), h->rowind.data());
    }
  } catch (const std::bad_alloc&) {
    return fail(h, SPB_ERR_OOM, "symbolic_from: host allocation failed");
  } catch (const std::exception& e) {
    return fail(h, SPB_ERR_STRUCTURE, e.what());
  }
  return install_device(h);
}

int spb_predict_device_bytes(const spb_handle* h, int32_t precision, int32_t nrhs, int64_t* bytes) {
  if (!h || !bytes || nrhs < 0 || (precision != SPB_PRECISION_FP64 && precision != SPB_PRECISION_FP32_IR))
    return SPB_ERR_INVALID;
  if (!h->have_symbolic) return SPB_ERR_STATE;
  *bytes = predict_bytes(h, precision == SPB_PRECISION_FP32_IR, nrhs);
  return SPB_OK;
}

int spb_replan(spb_handle* h, int32_t small_max_w, int32_t big_tile_rows, int32_t outer_nb) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic) return fail(h, SPB_ERR_STATE, "replan: no symbolic analysis");
  if (small_max_w < 0 || small_max_w > 64 || big_tile_rows < 0 || outer_nb < 0 || outer_nb > 4096 || outer_nb % 64)
    return fail(h, SPB_ERR_INVALID,
                "replan: small_max_w must be in [0, 64], big_tile_rows >= 0, outer_nb a multiple of 64 in [0, 4096]");
  h->opt.plan_small_max_w = small_max_w;
  h->opt.plan_big_tile_rows = big_tile_rows;
  h->opt.plan_outer_nb = outer_nb;
  if (h->device >= 0) {
    SPB_CK(h, cudaSetDevice(h->device));
    release_device(h);
  }
  h->have_symbolic = h->have_values = h->factored = h->have_solution = false;
  return install_symbolic(h, h->sym.n, h->colptr.data(), h->rowind.data());
}

int spb_symbolic_batch(spb_handle* h, int32_t nsys, const int32_t* sys_offsets, int32_t n, const int64_t* colptr,
                       const int32_t* rowind) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (nsys <= 0 || !sys_offsets) return fail(h, SPB_ERR_INVALID, "symbolic_batch: no systems");
  if (h->opt.ordering == SPB_ORDERING_USER)
    return fail(h, SPB_ERR_INVALID, "symbolic_batch: USER ordering is per matrix; use MMD, AMD, RCM or NATURAL");
  int rc = begin_symbolic(h, n, colptr, rowind);
  if (rc) return rc;
  if (sys_offsets[0] != 0 || sys_offsets[nsys] != n) return fail(h, SPB_ERR_INVALID, "symbolic_batch: bad offsets");
  for (int k = 0; k < nsys; ++k)
    if (sys_offsets[k + 1] <= sys_offsets[k]) return fail(h, SPB_ERR_INVALID, "symbolic_batch: empty system");
  // each system's columns may only hold rows of the same system (block-diagonal matrix)
  for (int k = 0; k < nsys; ++k)
    for (int c = sys_offsets[k] + 1; c <= sys_offsets[k + 1]; ++c)
      for (int64_t p = colptr[c - 1]; p < colptr[c]; ++p)
        if (rowind[p - 1] > sys_offsets[k + 1])
          return fail(h, SPB_ERR_INVALID, "symbolic_batch: entry couples two systems");
  std::vector<spb::Symbolic> parts(nsys);
  std::vector<std::string> errors(nsys);
  const spb::RelaxParams rp = relax_of(h->opt);
  const spb::OrderingKind ord = (spb::OrderingKind)h->opt.ordering;
  // largest systems first, so that no large analysis starts last and runs alone
  std::vector<int> order(nsys);
  for (int k = 0; k < nsys; ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    const int64_t ex = colptr[sys_offsets[x + 1]] - colptr[sys_offsets[x]];
    const int64_t ey = colptr[sys_offsets[y + 1]] - colptr[sys_offsets[y]];
    return ex > ey;
  });
  std::atomic<int> next{0};
  auto worker = [&]() {
    std::vector<int64_t> cp;
    std::vector<int32_t> ri;
    for (int slot = next++; slot < nsys; slot = next++) {
      const int k = order[slot];
      const int o = sys_offsets[k], nk = sys_offsets[k + 1] - o;
      const int64_t p0 = colptr[o];
      cp.assign(nk + 1, 0);
      for (int c = 0; c <= nk; ++c) cp[c] = colptr[o + c] - p0 + 1;
      ri.resize(cp[nk] - 1);
      for (int64_t p = 0; p < cp[nk] - 1; ++p) ri[p] = rowind[p0 - 1 + p] - o;
      try {
        parts[k] = spb::symbolic_factorization(nk, cp.data(), ri.data(), ord, rp);
      } catch (const std::exception& e) {
        errors[k] = e.what();
      }
    }
  };
  unsigned nthreads = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), (unsigned)nsys));
  std::vector<std::thread> pool;
  for (unsigned t = 0; t + 1 < nthreads; ++t) pool.emplace_back(worker);
  worker();
  for (std::thread& t : pool) t.join();
  for (int k = 0; k < nsys; ++k)
    if (!errors[k].empty())
      return fail(h, SPB_ERR_INVALID, "symbolic_batch: system " + std::to_string(k) + ": " + errors[k]);
  try {
    h->sym = spb::merge_symbolic(parts);
  } catch (const std::exception& e) {
    return fail(h, SPB_ERR_INVALID, e.what());
  }
  if (nsys > 1) h->seg_off.assign(sys_offsets, sys_offsets + nsys + 1);
  return install_symbolic(h, n, colptr, rowind);
}

static int distribute_common(spb_handle* h) {
  const spb::Plan& P = h->plan;
  SPB_CK(h, cudaMemsetAsync(h->dL, 0, (size_t)P.arena_elems * h->elem, h->stream));
  if (h->ldl) SPB_CK(h, cudaMemsetAsync(h->dW, 0, (size_t)P.arena_elems * sizeof(double), h->stream));
  SPB_CK(h, cudaMemsetAsync(h->dstatus, 0, sizeof(Status), h->stream));
  if (h->profiling) {
    SPB_CK(h, ensure_events(h, 2));
    SPB_CK(h, cudaEventRecord(h->events[0], h->stream));
  }
  spb::dev::launch_assemble(h->stream, h->dL, h->fp32, h->damap, h->dA, h->nnz_a);
  if (h->fp32) {  // FP64 copy of A for the refinement residuals, and ||A||_inf
    spb::dev::launch_gather(h->stream, h->d_val, h->dA, h->d_csrsrc, (int64_t)h->csr_col.size());
    SPB_CK(h, cudaMemsetAsync(h->d_norms + 1, 0, sizeof(double) * num_segments(h), h->stream));
    spb::dev::launch_rowsum_segmax(h->stream, h->d_rowptr, h->d_val, h->sym.n, h->d_rowseg, h->d_norms + 1);
  }
  SPB_CK(h, cudaGetLastError());
  if (h->profiling) SPB_CK(h, cudaEventRecord(h->events[1], h->stream));
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  if (h->profiling) {
    float ms = 0.f;
    SPB_CK(h, cudaEventElapsedTime(&ms, h->events[0], h->events[1]));
    clear_kinds(h, SPB_KIND_ASSEMBLE, SPB_KIND_ASSEMBLE);
    h->prof.ms[SPB_KIND_ASSEMBLE] = ms;
    h->prof.bytes[SPB_KIND_ASSEMBLE] = (double)h->nnz_a * 24.0;  // value + index read, value written
    h->prof.launches[SPB_KIND_ASSEMBLE] = 1;
  }
  h->have_values = true;
  h->factored = h->have_solution = false;
  return SPB_OK;
}

int spb_distribute(spb_handle* h, const double* nzval) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (h->device < 0) return fail(h, SPB_ERR_STATE, "host-only handle (device < 0) has no numeric phase");
  if (!h->have_symbolic) return fail(h, SPB_ERR_STATE, "distribute: call spb_symbolic first");
  if (!nzval) return fail(h, SPB_ERR_INVALID, "distribute: null values");
  SPB_CK(h, cudaSetDevice(h->device));
  SPB_CK(h, cudaMemcpyAsync(h->dA, nzval, h->nnz_a * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  return distribute_common(h);
}

int spb_distribute_device(spb_handle* h, const double* d_nzval) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (h->device < 0) return fail(h, SPB_ERR_STATE, "host-only handle (device < 0) has no numeric phase");
  if (!h->have_symbolic) return fail(h, SPB_ERR_STATE, "distribute: call spb_symbolic first");
  if (!d_nzval) return fail(h, SPB_ERR_INVALID, "distribute: null values");
  SPB_CK(h, cudaSetDevice(h->device));
  SPB_CK(h, cudaMemcpyAsync(h->dA, d_nzval, h->nnz_a * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  return distribute_common(h);
}

int spb_factorize(spb_handle* h) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (h->device < 0) return fail(h, SPB_ERR_STATE, "host-only handle (device < 0) has no numeric phase");
  if (!h->have_values) return fail(h, SPB_ERR_STATE, "factorize: call spb_distribute first");
  if (h->factored) return fail(h, SPB_ERR_STATE, "factorize: values already factored; distribute again");
  SPB_CK(h, cudaSetDevice(h->device));
  h->trace_fresh = false;
  if (h->profiling) {
    int rc = factor_profiled(h);
    if (rc) return rc;
  } else if (!h->fgraph && !h->plan.steps.empty()) {
    cudaGraph_t g;
    SPB_CK(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t qe = enqueue_factor(h);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (qe != cudaSuccess) {
      if (e == cudaSuccess) cudaGraphDestroy(g);
      return cuda_fail(h, qe, "factorize: graph capture");
    }
    if (e != cudaSuccess) return cuda_fail(h, e, "factorize: graph capture");
    e = cudaGraphInstantiate(&h->fgraph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(h, e, "factorize: graph instantiate");
  }
  if (h->fgraph && !h->profiling) SPB_CK(h, cudaGraphLaunch(h->fgraph, h->stream));
  Status st;
  SPB_CK(h, cudaMemcpyAsync(&st, h->dstatus, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  h->factored = true;
  h->inv_stale = true;
  if (st.code == 1) {
    char msg[128];
    if (h->ldl)
      snprintf(msg, sizeof msg, "LDL^T: zero pivot in supernode %d, column %d", st.supernode + 1, st.column + 1);
    else
      snprintf(msg, sizeof msg, "Matrix is not HPD: non-positive pivot in supernode %d, column %d", st.supernode + 1,
               st.column + 1);
    return fail(h, SPB_ERR_NOT_SPD, msg);
  }
  if (st.code == 3) {  // a bounded wait of the persistent factorization expired; the context is intact
    SPB_CK(h, cudaMemsetAsync(h->dstatus, 0, sizeof(Status), h->stream));
    SPB_CK(h, cudaStreamSynchronize(h->stream));
    h->factored = false;
    return fail(h, SPB_ERR_TIMEOUT, "factorize: a device wait expired");
  }
  if (st.code != 0) return fail(h, SPB_ERR_STRUCTURE, "factorize: update row missing from target structure");
  h->trace_fresh = h->factor_trace && !h->profiling && persistent_factor(h) && !h->plan.ftasks.empty();
  return SPB_OK;
}

int spb_solve_device(spb_handle* h, const double* d_rhs, double* d_x, int32_t nrhs, int64_t ld) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (h->device < 0) return fail(h, SPB_ERR_STATE, "host-only handle (device < 0) has no numeric phase");
  if (!h->factored) return fail(h, SPB_ERR_STATE, "solve: call spb_factorize first");
  const int n = h->sym.n;
  if (nrhs <= 0 || ld < n || !d_rhs || !d_x) return fail(h, SPB_ERR_INVALID, "solve: bad right-hand side");
  SPB_CK(h, cudaSetDevice(h->device));
  int rc = ensure_rhs_capacity(h, nrhs);
  if (rc) return rc;
  if (h->fp32) return ir_solve(h, d_rhs, ld, d_x, ld, nrhs);
  if (h->profiling) SPB_CK(h, ensure_events(h, 4 * (size_t)((nrhs + 63) / 64) + 2));
  spb::dev::launch_permute_in(h->stream, h->dX, n, d_rhs, ld, h->dinvp0, n, nrhs);
  enqueue_solve(h, nrhs);
  rc = collect_solve_profile(h, nrhs);
  if (rc) return rc;
  spb::dev::launch_permute_out(h->stream, d_x, ld, h->dX, n, h->dinvp0, n, nrhs);
  SPB_CK(h, cudaGetLastError());
  return check_solve_status(h);
}

int spb_solve(spb_handle* h, const double* rhs, int32_t nrhs, int64_t ldb) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (h->device < 0) return fail(h, SPB_ERR_STATE, "host-only handle (device < 0) has no numeric phase");
  if (!h->factored) return fail(h, SPB_ERR_STATE, "solve: call spb_factorize first");
  const int n = h->sym.n;
  if (nrhs <= 0 || ldb < n || !rhs) return fail(h, SPB_ERR_INVALID, "solve: bad right-hand side");
  SPB_CK(h, cudaSetDevice(h->device));
  int rc = ensure_rhs_capacity(h, nrhs);
  if (rc) return rc;
  SPB_CK(h, cudaMemcpy2DAsync(h->dB, (size_t)n * 8, rhs, (size_t)ldb * 8, (size_t)n * 8, nrhs, cudaMemcpyHostToDevice,
                              h->stream));
  if (h->fp32) {
    rc = ir_solve(h, h->dB, n, h->dXo, n, nrhs);
    if (rc) return rc;
    h->have_solution = true;
    h->x_nrhs = nrhs;
    return SPB_OK;
  }
  if (h->profiling) SPB_CK(h, ensure_events(h, 4 * (size_t)((nrhs + 63) / 64)));
  spb::dev::launch_permute_in(h->stream, h->dX, n, h->dB, n, h->dinvp0, n, nrhs);
  enqueue_solve(h, nrhs);
  rc = collect_solve_profile(h, nrhs);
  if (rc) return rc;
  SPB_CK(h, cudaGetLastError());
  rc = check_solve_status(h);
  if (rc) return rc;
  h->have_solution = true;
  h->x_nrhs = nrhs;
  return SPB_OK;
}

int spb_get_solution(spb_handle* h, double* B, int32_t nrhs, int64_t ldb) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (h->device < 0) return fail(h, SPB_ERR_STATE, "host-only handle (device < 0) has no numeric phase");
  if (!h->have_solution) return fail(h, SPB_ERR_STATE, "get_solution: call spb_solve first");
  const int n = h->sym.n;
  if (!B || nrhs <= 0 || nrhs > h->x_nrhs || ldb < n) return fail(h, SPB_ERR_INVALID, "get_solution: bad output");
  SPB_CK(h, cudaSetDevice(h->device));
  const double* src = h->dXo;  // refined solution, original order
  if (!h->fp32) {
    spb::dev::launch_permute_out(h->stream, h->dB, n, h->dX, n, h->dinvp0, n, nrhs);
    src = h->dB;
  }
  SPB_CK(h, cudaMemcpy2DAsync(B, (size_t)ldb * 8, src, (size_t)n * 8, (size_t)n * 8, nrhs, cudaMemcpyDeviceToHost,
                              h->stream));
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  return SPB_OK;
}

int spb_get_info(spb_handle* h, spb_info* info) {
  if (check_handle(h) || !info) return SPB_ERR_INVALID;
  if (!h->have_symbolic) return fail(h, SPB_ERR_STATE, "info: no symbolic factorization");
  std::memset(info, 0, sizeof(*info));
  const spb::Plan& P = h->plan;
  if (!h->cells_built) {
    h->cells = spb::build_cells(h->sym);
    h->cells_built = true;
  }
  info->n = h->sym.n;
  info->nsuper = P.nsuper;
  info->nlevels = P.nlevels;
  int mw = 0;
  for (const auto& m : P.meta) mw = std::max(mw, m.w);
  info->max_width = mw;
  info->nnz_a = h->nnz_a;
  info->nnz_l = h->sym.nnzL_stat;
  info->lindx_size = (int64_t)h->sym.lindx.size();
  info->arena_bytes = P.arena_elems * 8;
  info->device_bytes = h->device_bytes;
  info->flops_stat = h->sym.flops_stat;
  info->flops_exec = P.exec_flops;
  info->ncells = (int32_t)h->cells.cells.size();
  info->nblocks = (int32_t)h->cells.block_first_row.size();
  info->factor_launches = persistent_factor(h) ? 1 : (int32_t)P.steps.size();
  info->dense_root_width = 0;  // the cluster root solve gave way to the super-block solve
  info->factor_sched_us = P.fsim_us;
  info->factor_tasks = (int32_t)P.ftasks.size();
  info->inverse_bytes = P.inv_elems * (int64_t)(h->opt.precision == SPB_PRECISION_FP32_IR ? 4 : 8);
  info->ir_iterations = h->ir_iterations;
  info->backward_error = h->backward_error;
  return SPB_OK;
}

int spb_get_ordering(spb_handle* h, int32_t* perm, int32_t* invp) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic) return fail(h, SPB_ERR_STATE, "no symbolic factorization");
  if (perm) std::copy(h->sym.perm.begin(), h->sym.perm.end(), perm);
  if (invp) std::copy(h->sym.invp.begin(), h->sym.invp.end(), invp);
  return SPB_OK;
}

int spb_get_mmd_invp(spb_handle* h, int32_t* invp) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic) return fail(h, SPB_ERR_STATE, "no symbolic factorization");
  if (invp) std::copy(h->sym.mmd_invp.begin(), h->sym.mmd_invp.end(), invp);
  return SPB_OK;
}

int spb_get_etree(spb_handle* h, int32_t* parent) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic) return fail(h, SPB_ERR_STATE, "no symbolic factorization");
  if (parent) std::copy(h->sym.parent.begin(), h->sym.parent.end(), parent);
  return SPB_OK;
}

int spb_get_colcounts(spb_handle* h, int32_t* cc_fund, int32_t* cc_relaxed) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic) return fail(h, SPB_ERR_STATE, "no symbolic factorization");
  if (cc_fund) std::copy(h->sym.cc_fund.begin(), h->sym.cc_fund.end(), cc_fund);
  if (cc_relaxed) std::copy(h->sym.cc.begin(), h->sym.cc.end(), cc_relaxed);
  return SPB_OK;
}

int spb_get_supernodes(spb_handle* h, int32_t* xsuper, int32_t* supmember) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic) return fail(h, SPB_ERR_STATE, "no symbolic factorization");
  if (xsuper) std::copy(h->sym.xsuper.begin(), h->sym.xsuper.end(), xsuper);
  if (supmember) std::copy(h->sym.supmember.begin(), h->sym.supmember.end(), supmember);
  return SPB_OK;
}

int spb_get_structure(spb_handle* h, int64_t* xlindx, int32_t* lindx) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic) return fail(h, SPB_ERR_STATE, "no symbolic factorization");
  if (xlindx) std::copy(h->sym.xlindx.begin(), h->sym.xlindx.end(), xlindx);
  if (lindx) std::copy(h->sym.lindx.begin(), h->sym.lindx.end(), lindx);
  return SPB_OK;
}

int spb_get_cells(spb_handle* h, int32_t* cI, int32_t* cK, int32_t* cnr, int32_t* cfb, int32_t* cnb, int32_t* bfr,
                  int32_t* bnr) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic) return fail(h, SPB_ERR_STATE, "no symbolic factorization");
  if (!h->cells_built) {
    h->cells = spb::build_cells(h->sym);
    h->cells_built = true;
  }
  const auto& C = h->cells;
  for (size_t i = 0; i < C.cells.size(); ++i) {
    if (cI) cI[i] = C.cells[i].I;
    if (cK) cK[i] = C.cells[i].K;
    if (cnr) cnr[i] = C.cells[i].nrows;
    if (cfb) cfb[i] = C.cells[i].first_block;
    if (cnb) cnb[i] = C.cells[i].nblocks;
  }
  if (bfr) std::copy(C.block_first_row.begin(), C.block_first_row.end(), bfr);
  if (bnr) std::copy(C.block_nrows.begin(), C.block_nrows.end(), bnr);
  return SPB_OK;
}

int spb_get_factor(spb_handle* h, double* out) {
  if (check_handle(h) || !out) return SPB_ERR_INVALID;
  if (h->device < 0) return fail(h, SPB_ERR_STATE, "host-only handle (device < 0) has no numeric phase");
  if (!h->factored) return fail(h, SPB_ERR_STATE, "get_factor: call spb_factorize first");
  SPB_CK(h, cudaSetDevice(h->device));
  const spb::Plan& P = h->plan;
  std::vector<double> arena(P.arena_elems);
  if (h->fp32) {
    std::vector<float> a32(P.arena_elems);
    SPB_CK(h, cudaMemcpy(a32.data(), h->dL, P.arena_elems * sizeof(float), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < P.arena_elems; ++i) arena[i] = a32[i];
  } else {
    SPB_CK(h, cudaMemcpy(arena.data(), h->dL, P.arena_elems * sizeof(double), cudaMemcpyDeviceToHost));
  }
  std::vector<double> warena;  // LDL^T: D from the diagonal of L D
  if (h->ldl) {
    warena.resize(P.arena_elems);
    SPB_CK(h, cudaMemcpy(warena.data(), h->dW, P.arena_elems * sizeof(double), cudaMemcpyDeviceToHost));
  }
  int64_t pos = 0;
  for (const auto& m : P.meta) {
    for (int c = 0; c < m.w; ++c)
      for (int r = 0; r < m.h; ++r) {
        const int64_t at = m.off + r + (int64_t)c * m.ld;
        out[pos + r + (int64_t)c * m.h] = (r < c) ? 0.0 : (r == c && h->ldl) ? warena[at] : arena[at];
      }
    pos += (int64_t)m.h * m.w;
  }
  return SPB_OK;
}

int spb_set_wait_limit(spb_handle* h, int64_t polls) {
  if (check_handle(h) || polls <= 0) return SPB_ERR_INVALID;
  h->wait_limit = polls;
  return SPB_OK;
}

int spb_debug_stall(spb_handle* h, int32_t supernode) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic || h->device < 0) return fail(h, SPB_ERR_STATE, "debug_stall: needs a device handle");
  const int ns = h->plan.nsuper;
  if (supernode >= ns) return fail(h, SPB_ERR_INVALID, "debug_stall: supernode out of range");
  std::vector<int32_t> e = h->plan.fwd_pending;
  if (supernode >= 0) e[supernode] += 1;
  SPB_CK(h, cudaMemcpyAsync(h->dexpected, e.data(), e.size() * 4, cudaMemcpyHostToDevice, h->stream));
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  h->stall_supernode = supernode;
  return SPB_OK;
}

int spb_set_factor_trace(spb_handle* h, int32_t on) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic || h->device < 0) return fail(h, SPB_ERR_STATE, "factor_trace: needs a device handle");
  SPB_CK(h, cudaSetDevice(h->device));
  if (on && !h->dftrace) {
    SPB_CK(h, dalloc(h, &h->dftrace, 4 * std::max<size_t>(1, h->plan.ftasks.size())));
    SPB_CK(h, cudaStreamSynchronize(h->own_stream));
  }
  if (h->fgraph) {  // the captured factorization holds the trace pointer: capture again
    cudaGraphExecDestroy(h->fgraph);
    h->fgraph = nullptr;
  }
  h->factor_trace = on != 0;
  return SPB_OK;
}

int spb_get_factor_trace(spb_handle* h, uint64_t* out, int64_t cap, int64_t* ntasks, int32_t* kinds) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->dftrace) return fail(h, SPB_ERR_STATE, "factor_trace: no traced factorization");
  const int64_t n = (int64_t)h->plan.ftasks.size();
  if (ntasks) *ntasks = n;
  if (!out) return SPB_OK;
  if (cap < n) return fail(h, SPB_ERR_INVALID, "factor_trace: buffer too small");
  SPB_CK(h, cudaMemcpy(out, h->dftrace, 4 * n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  if (kinds)
    for (int64_t i = 0; i < n; ++i) kinds[i] = h->plan.ftasks[i].kind;
  return SPB_OK;
}

int spb_reorder_factor_from_trace(spb_handle* h) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic || h->device < 0) return fail(h, SPB_ERR_STATE, "reorder: needs an analysed device handle");
  if (!persistent_factor(h) || h->plan.ftasks.empty())
    return fail(h, SPB_ERR_STATE, "reorder: the factorization does not use the persistent schedule");
  if (!h->trace_fresh || !h->dftrace)
    return fail(h, SPB_ERR_STATE, "reorder: factorize once with spb_set_factor_trace(h, 1) first");
  SPB_CK(h, cudaSetDevice(h->device));
  spb::Plan& P = h->plan;
  const size_t n = P.ftasks.size();
  std::vector<unsigned long long> tr(4 * n);
  SPB_CK(h, cudaMemcpy(tr.data(), h->dftrace, tr.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  std::vector<double> us(n);
  for (size_t i = 0; i < n; ++i) {  // dependencies met -> done, nanoseconds of the global timer
    const unsigned long long met = tr[4 * i + 1], done = tr[4 * i + 2];
    us[i] = done > met ? (double)(done - met) * 1e-3 : 0.0;
  }
  try {
    spb::reorder_factor_tasks(P, plan_params_of(h->opt), us);
  } catch (const std::exception& e) {
    return fail(h, SPB_ERR_INVALID, e.what());
  }
  // same sizes: the arrays are rewritten in place, so a captured factorization stays valid
  SPB_CK(h, cudaMemcpyAsync(h->dftasks, P.ftasks.data(), n * sizeof(spb::FTask), cudaMemcpyHostToDevice, h->stream));
  SPB_CK(h, cudaMemcpyAsync(h->dfwaits, P.fwaits.data(), P.fwaits.size() * sizeof(spb::FWait), cudaMemcpyHostToDevice,
                            h->stream));
  SPB_CK(h, cudaMemcpyAsync(h->dfsigs, P.fsigs.data(), P.fsigs.size() * 4, cudaMemcpyHostToDevice, h->stream));
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  h->trace_fresh = false;
  return SPB_OK;
}

int spb_debug_stall_factor(spb_handle* h, int32_t supernode) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic || h->device < 0) return fail(h, SPB_ERR_STATE, "debug_stall_factor: needs a device handle");
  if (supernode >= h->plan.nsuper) return fail(h, SPB_ERR_INVALID, "debug_stall_factor: supernode out of range");
  std::vector<spb::FWait> w = h->plan.fwaits;
  for (spb::FWait& x : w)
    if (supernode >= 0 && x.ctr == supernode) x.target += 1;  // ext counters come first
  std::vector<spb::FTask> t = h->plan.ftasks;  // and the tasks' copies of their first wait
  for (spb::FTask& x : t)
    if (supernode >= 0 && x.nwait > 0 && x.w0_ctr == supernode) x.w0_target += 1;
  SPB_CK(h, cudaMemcpyAsync(h->dfwaits, w.data(), w.size() * sizeof(spb::FWait), cudaMemcpyHostToDevice, h->stream));
  SPB_CK(h, cudaMemcpyAsync(h->dftasks, t.data(), t.size() * sizeof(spb::FTask), cudaMemcpyHostToDevice, h->stream));
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  return SPB_OK;
}

int spb_clear_status(spb_handle* h) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (!h->have_symbolic || h->device < 0) return fail(h, SPB_ERR_STATE, "clear_status: needs a device handle");
  SPB_CK(h, cudaMemsetAsync(h->dstatus, 0, sizeof(Status), h->stream));
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  return SPB_OK;
}

int spb_set_stream(spb_handle* h, void* stream) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (h->device < 0) return fail(h, SPB_ERR_STATE, "host-only handle (device < 0) has no stream");
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return SPB_OK;
}

int spb_get_solve_trace(spb_handle* h, int32_t sweep, uint64_t* out, int64_t cap, int64_t* ntasks) {
  if (check_handle(h) || !ntasks || (sweep != 0 && sweep != 1)) return SPB_ERR_INVALID;
  const spb::Plan& P = h->plan;
  const size_t nt = sweep == 0 ? P.fwd_tasks.size() : P.bwd_tasks.size();
  *ntasks = (int64_t)nt;
  if (!h->dtrace) return fail(h, SPB_ERR_STATE, "solve_trace: no profiled solve yet");
  if (!out) return SPB_OK;
  const size_t n = std::min(nt, (size_t)std::max<int64_t>(cap, 0));
  SPB_CK(h, cudaSetDevice(h->device));
  SPB_CK(h, cudaStreamSynchronize(h->stream));
  SPB_CK(h, cudaMemcpy(out, h->dtrace + (sweep ? 4 * P.fwd_tasks.size() : 0), 4 * n * sizeof(uint64_t),
                       cudaMemcpyDeviceToHost));
  return SPB_OK;
}

int spb_set_profiling(spb_handle* h, int on) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  h->profiling = on != 0;
  return SPB_OK;
}

int spb_get_profile(spb_handle* h, spb_profile* out) {
  if (check_handle(h) || !out) return SPB_ERR_INVALID;
  *out = h->prof;
  return SPB_OK;
}

int spb_get_status(spb_handle* h, int32_t* code, int32_t* supernode, int32_t* column) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (h->device < 0) return fail(h, SPB_ERR_STATE, "host-only handle (device < 0) has no numeric phase");
  if (!h->have_symbolic) return fail(h, SPB_ERR_STATE, "no symbolic factorization");
  SPB_CK(h, cudaSetDevice(h->device));
  Status st;
  SPB_CK(h, cudaMemcpy(&st, h->dstatus, sizeof(st), cudaMemcpyDeviceToHost));
  if (code) *code = st.code;
  if (supernode) *supernode = st.supernode;
  if (column) *column = st.column;
  return SPB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free solve.
//
// spb_solve_device lazily grows the handle's right-hand-side workspace with
// cudaMalloc when a call asks for more right-hand sides than before.  Some
// callers cannot let that happen: services that reserve their device-memory
// budget up front (another allocator owns the rest of the GPU, so an allocation
// in mid-request could fail), and latency-critical callers for which cudaMalloc
// and cudaFree may synchronize the device.  spb_solve_device_noalloc
// gives them the same solve with its scratch (permuted right-hand sides, the
// forward solution and the dependency counters of the persistent sweeps) in one file-scope
// __device__ array, so no call allocates or frees anything.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocXBytes = (size_t)32 << 20;   // permuted right-hand sides: 4 Mi doubles
constexpr size_t kNoAllocSyncBytes = (size_t)1 << 20; // counters of the sweeps: 256 Ki int32
constexpr int kNoAllocMaxDevices = 64;

// Held by every GPU that loads this library until the process exits (65 MiB): the
// permuted right-hand sides X, the forward solution Z (same size) and the counters.
static __device__ __align__(256) unsigned char g_noalloc_scratch[2 * kNoAllocXBytes + kNoAllocSyncBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kNoAllocMaxDevices] = {};  // device address of g_noalloc_scratch, per device

// Host code must not use g_noalloc_scratch's name as a device address: on the
// host it is a stand-in.  Resolve the real address once per device, with that
// device current.
int noalloc_scratch(spb_handle* h, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[h->device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_fail(h, e == cudaSuccess ? cudaErrorInvalidSymbol : e,
                                                 "solve_noalloc: cudaGetSymbolAddress");
    g_noalloc_addr[h->device] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_addr[h->device]);
  return SPB_OK;
}

}  // namespace

extern "C" int spb_solve_device_noalloc(spb_handle* h, const double* d_rhs, double* d_x, int32_t nrhs, int64_t ld) {
  if (check_handle(h)) return SPB_ERR_INVALID;
  if (h->device < 0) return fail(h, SPB_ERR_STATE, "host-only handle (device < 0) has no numeric phase");
  if (!h->factored) return fail(h, SPB_ERR_STATE, "solve: call spb_factorize first");
  const int n = h->sym.n;
  if (nrhs <= 0 || ld < n || !d_rhs || !d_x) return fail(h, SPB_ERR_INVALID, "solve: bad right-hand side");
  if (h->device >= kNoAllocMaxDevices) return fail(h, SPB_ERR_INVALID, "solve_noalloc: device ordinal >= 64");
  if (h->fp32) return fail(h, SPB_ERR_STATE, "solve_noalloc: refinement (FP32_IR) needs workspace; use spb_solve_device");
  if ((size_t)n * (size_t)nrhs * sizeof(double) > kNoAllocXBytes) {
    char msg[160];
    snprintf(msg, sizeof msg, "solve_noalloc: n * nrhs = %lld exceeds the %zu right-hand-side entries of the "
             "static scratch (2 x 32 MiB)", (long long)n * nrhs, kNoAllocXBytes / sizeof(double));
    return fail(h, SPB_ERR_INVALID, msg);
  }
  if (spb::solve_sync_ints(h->plan) * sizeof(int32_t) > kNoAllocSyncBytes)
    return fail(h, SPB_ERR_INVALID,
                "solve_noalloc: 2 + 3 * supernodes + 2 * (64-column blocks) exceeds the 262,144 counters of the "
                "static scratch");
  SPB_CK(h, cudaSetDevice(h->device));
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(h, &base);
  if (rc) return rc;
  double* X = reinterpret_cast<double*>(base);
  double* Z = reinterpret_cast<double*>(base + kNoAllocXBytes);
  int32_t* sync = reinterpret_cast<int32_t*>(base + 2 * kNoAllocXBytes);
  spb::dev::launch_permute_in(h->stream, X, n, d_rhs, ld, h->dinvp0, n, nrhs);
  ensure_inverses(h);  // the first solve after a factorization computes them (arena of the analysis)
  enqueue_sweeps(h, X, Z, sync, nrhs, false);
  spb::dev::launch_permute_out(h->stream, d_x, ld, X, n, h->dinvp0, n, nrhs);
  SPB_CK(h, cudaGetLastError());
  return check_solve_status(h);
}
