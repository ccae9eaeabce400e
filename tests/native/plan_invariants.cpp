// Host-side invariants of the device plan (plan.cpp), checked on grid matrices and a
// block-diagonal batch without a GPU: tile shapes the tile engines rely on, the dispatch order of the persistent
// factorization (every task's dependencies are signalled by tasks handed out before it),
// and the tiny-leaf solve tasks.  Prints "ok" or the first violation and exits non-zero.
#include <cstdio>
#include <algorithm>
#include <cstdlib>
#include <map>
#include <set>
#include <vector>

#include "plan.hpp"

using namespace spb;

static int fails = 0;
static long long n_tiles = 0, n_ftasks = 0, n_tiny = 0, n_big_tiles = 0;
#define CHECK(cond, ...)                  \
  do {                                    \
    if (!(cond)) {                        \
      if (fails++ < 10) {                 \
        std::fprintf(stderr, __VA_ARGS__); \
        std::fprintf(stderr, "\n");       \
      }                                   \
    }                                     \
  } while (0)

// Lower CSC (1-based, diagonal first) of a k x k x k grid with 7- or 27-point couplings.
static void grid_matrix(int k, bool full, std::vector<int64_t>& cp, std::vector<int32_t>& ri) {
  const int n = k * k * k;
  cp.assign(1, 1);
  ri.clear();
  for (int z = 0; z < k; ++z)
    for (int y = 0; y < k; ++y)
      for (int x = 0; x < k; ++x) {
        const int c = x + k * (y + k * z);
        std::set<int> rows{c};
        for (int dz = -1; dz <= 1; ++dz)
          for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
              const int nn = (dx != 0) + (dy != 0) + (dz != 0);
              if (nn == 0 || (!full && nn != 1)) continue;
              const int X = x + dx, Y = y + dy, Z = z + dz;
              if (X < 0 || Y < 0 || Z < 0 || X >= k || Y >= k || Z >= k) continue;
              const int r = X + k * (Y + k * Z);
              if (r > c) rows.insert(r);
            }
        for (int r : rows) ri.push_back(r + 1);
        cp.push_back((int64_t)ri.size() + 1);
      }
  (void)n;
}

// Lower CSC (1-based) of a dense n x n matrix: one supernode of n columns.
static void dense_matrix(int n, std::vector<int64_t>& cp, std::vector<int32_t>& ri) {
  cp.assign(1, 1);
  ri.clear();
  for (int c = 0; c < n; ++c) {
    for (int r = c; r < n; ++r) ri.push_back(r + 1);
    cp.push_back((int64_t)ri.size() + 1);
  }
}

// Lower CSC (1-based) of a path graph (tridiagonal): a chain of narrow supernodes.
static void path_matrix(int n, std::vector<int64_t>& cp, std::vector<int32_t>& ri) {
  cp.assign(1, 1);
  ri.clear();
  for (int c = 0; c < n; ++c) {
    ri.push_back(c + 1);
    if (c + 1 < n) ri.push_back(c + 2);
    cp.push_back((int64_t)ri.size() + 1);
  }
}

static long long n_rel = 0;

static void check_plan(const Symbolic& sym, const PlanParams& prm, const char* what) {
  const Plan P = build_plan(sym, prm);
  // relative indices (filled by host threads on large plans): every group's positions
  // equal a merge of its rows with its target's from the start
  n_rel += (long long)P.rel.size();
  {
    std::vector<int32_t> src(P.groups.size(), -1);
    for (int s = 0; s < P.nsuper; ++s) {
      const SnMeta& m = P.meta[s];
      for (int r = m.w; r < m.h; ++r) {
        const int g = P.row_group[m.lidx + r];
        CHECK(g >= 0 && g < (int)P.groups.size(), "%s: off-diagonal row without a group", what);
        if (g >= 0 && g < (int)P.groups.size() && src[g] < 0) src[g] = s;
      }
    }
    bool bad = false;
    for (size_t g = 0; g < P.groups.size() && !bad; ++g) {
      const RelGroup& gr = P.groups[g];
      if (src[g] < 0) { bad = true; break; }
      const SnMeta& m = P.meta[src[g]];
      const SnMeta& mt = P.meta[gr.t];
      const int32_t* rl = P.rows.data() + m.lidx;
      const int32_t* tl = P.rows.data() + mt.lidx;
      int q = 0;
      for (int i = gr.j0; i < m.h && !bad; ++i) {
        while (q < mt.h && tl[q] < rl[i]) ++q;
        bad = q == mt.h || tl[q] != rl[i] || P.rel[gr.rel_off + (i - gr.j0)] != q;
      }
    }
    CHECK(!bad, "%s: relative indices differ from a merge of the row lists", what);
  }
  // tiles
  for (const Step& st : P.steps) {
    if (st.kind != StepKind::Gemm) continue;
    for (int i = st.begin; i < st.begin + st.count; ++i) {
      const TileItem& t = P.tile_items[i];
      const SnMeta& m = P.meta[t.s];
      ++n_tiles;
      n_big_tiles += st.tile == 128;
      CHECK(t.mrows >= 1 && t.ncols >= 1 && t.kn >= 1, "%s: empty tile", what);
      CHECK(t.a_row0 >= 0 && t.a_row0 + t.mrows <= m.h && t.b_row0 >= 0 && t.b_row0 + t.ncols <= m.h,
            "%s: tile outside the panel rows", what);
      CHECK(t.k0 >= 0 && t.k0 + t.kn <= m.w, "%s: K range outside the panel", what);
      if (t.mode == 1) CHECK(t.a_row0 >= m.w && t.b_row0 >= m.w, "%s: external tile in the diagonal block", what);
      else CHECK(t.b_row0 >= t.k0 + t.kn && t.a_row0 >= t.k0 + t.kn, "%s: in-panel tile overlaps its K columns", what);
      if (st.tile == 128 && !prm.fp32)  // bulk copies start on the even row below
        CHECK((t.a_row0 & 1) + t.mrows <= 128 && (t.b_row0 & 1) + t.ncols <= 64, "%s: FP64 tile shape", what);
      if (st.tile == 128 && prm.fp32)   // 32-column TMA chunks that never read past the K range inside the panel
        CHECK(t.mrows <= 128 && t.ncols <= 128 && t.k0 % 4 == 0 && (t.kn % 32 == 0 || t.k0 + t.kn == m.w),
              "%s: FP32 tile shape", what);
      if (st.tile == 64) CHECK(t.mrows <= 64 && t.ncols <= 64, "%s: 64 x 64 tile shape", what);
    }
  }
  // persistent factorization: executing the tasks one by one in dispatch order never waits
  if (prm.factor_dag) {
    CHECK(!P.ftasks.empty(), "%s: no factor tasks", what);
    n_ftasks += (long long)P.ftasks.size();
    std::vector<int64_t> ctr(P.nfctr, 0);
    for (size_t i = 0; i < P.ftasks.size(); ++i) {
      const FTask& t = P.ftasks[i];
      CHECK(t.nwait == 0 || (t.w0_ctr == P.fwaits[t.wait0].ctr && t.w0_target == P.fwaits[t.wait0].target),
            "%s: task %zu's copy of its first wait differs from its wait list", what, i);
      for (int w = 0; w < t.nwait; ++w) {
        const FWait& fw = P.fwaits[t.wait0 + w];
        CHECK(fw.ctr >= 0 && fw.ctr < P.nfctr, "%s: wait on a counter out of range", what);
        CHECK(ctr[fw.ctr] >= fw.target, "%s: task %zu waits for a task handed out after it", what, i);
      }
      for (int q = 0; q < t.nsig; ++q) {
        const int c = P.fsigs[t.sig0 + q];
        CHECK(c >= 0 && c < P.nfctr, "%s: signal out of range", what);
        ++ctr[c];
      }
    }
  }
  // re-ordered by measured durations (here pseudo-random ones): the same tasks with the
  // same waits and signals, and again no task waits for one handed out after it
  if (prm.factor_dag) {
    Plan R = P;
    std::vector<double> us(R.ftasks.size());
    unsigned long long x = 88172645463325252ULL;
    for (double& u : us) {
      x ^= x << 13; x ^= x >> 7; x ^= x << 17;
      u = 0.5 + (double)(x % 100000) / 1000.0;
    }
    reorder_factor_tasks(R, prm, us);
    CHECK(R.ftasks.size() == P.ftasks.size() && R.fwaits.size() == P.fwaits.size() &&
          R.fsigs.size() == P.fsigs.size() && R.nfctr == P.nfctr, "%s: re-ordering changed the counts", what);
    auto key = [](const FTask& t) { return ((long long)(t.kind == 0 ? 0 : t.kind <= 2 ? 1 : 2) << 32) | t.item; };
    std::map<long long, size_t> pos;
    for (size_t i = 0; i < P.ftasks.size(); ++i) pos[key(P.ftasks[i])] = i;
    std::vector<int64_t> ctr(R.nfctr, 0);
    for (size_t i = 0; i < R.ftasks.size(); ++i) {
      const FTask& t = R.ftasks[i];
      auto it = pos.find(key(t));
      CHECK(it != pos.end(), "%s: re-ordering made a new task", what);
      if (it == pos.end()) continue;
      const FTask& o = P.ftasks[it->second];
      CHECK(o.kind == t.kind && o.nwait == t.nwait && o.nsig == t.nsig, "%s: re-ordered task differs", what);
      CHECK(t.nwait == 0 || (t.w0_ctr == R.fwaits[t.wait0].ctr && t.w0_target == R.fwaits[t.wait0].target),
            "%s: re-ordered task's copy of its first wait differs", what);
      for (int w = 0; w < t.nwait && o.nwait == t.nwait; ++w)
        CHECK(R.fwaits[t.wait0 + w].ctr == P.fwaits[o.wait0 + w].ctr &&
                  R.fwaits[t.wait0 + w].target == P.fwaits[o.wait0 + w].target,
              "%s: re-ordered task waits differ", what);
      for (int q = 0; q < t.nsig && o.nsig == t.nsig; ++q)
        CHECK(R.fsigs[t.sig0 + q] == P.fsigs[o.sig0 + q], "%s: re-ordered task signals differ", what);
      for (int w = 0; w < t.nwait; ++w) {
        const FWait& fw = R.fwaits[t.wait0 + w];
        CHECK(ctr[fw.ctr] >= fw.target, "%s: re-ordered task %zu waits for a task handed out after it", what, i);
      }
      for (int q = 0; q < t.nsig; ++q) ++ctr[R.fsigs[t.sig0 + q]];
      pos.erase(it);
    }
    CHECK(pos.empty(), "%s: re-ordering lost tasks", what);
  }
  // solve: tiny leaves first (forward) and last (backward), each in exactly one batch
  std::vector<int> seen(P.nsuper, 0);
  bool tiny_phase = true;
  for (const SolveTask& t : P.fwd_tasks) {
    if (t.kind == 6) {
      CHECK(tiny_phase, "%s: a tiny batch after other forward tasks", what);
      CHECK(t.t >= 1 && t.t <= kTinyBatch && t.i + t.t <= (int)P.tiny.size(), "%s: tiny batch range", what);
      for (int j = t.i; j < t.i + t.t; ++j) seen[P.tiny[j]]++;
    } else {
      tiny_phase = false;
      seen[t.s] += 0;
    }
  }
  n_tiny += (long long)P.tiny.size();
  for (int s : P.tiny) {
    const SnMeta& m = P.meta[s];
    CHECK(seen[s] == 1, "%s: tiny supernode %d in %d batches", what, s, seen[s]);
    CHECK(P.level[s] == 0 && m.w <= kTinyMaxW && (int64_t)m.w * m.h <= kTinyMaxElems, "%s: tiny criteria", what);
  }
  std::vector<int> fwd_tasks_of(P.nsuper, 0), bwd_tasks_of(P.nsuper, 0);
  for (const SolveTask& t : P.fwd_tasks)
    if (t.kind != 6) fwd_tasks_of[t.s]++;
  bool after = false;
  int bwd_tiny = 0;
  for (const SolveTask& t : P.bwd_tasks) {
    if (t.kind == 6) {
      after = true;
      bwd_tiny += t.t;
    } else {
      CHECK(!after, "%s: a backward task after the tiny batches", what);
      bwd_tasks_of[t.s]++;
    }
  }
  CHECK(bwd_tiny == (int)P.tiny.size(), "%s: backward tiny count", what);
  // forward arrivals: what the tasks signal (one per relative-index group of the rows of
  // each 64-row off-diagonal tile they scatter: O tasks per tile, F and tiny supernodes
  // per tile of all their rows) equals what each target waits for
  std::vector<int64_t> arrivals(P.nsuper, 0);
  auto signal_rows = [&](int s, int r0, int r1) {
    const SnMeta& m = P.meta[s];
    const int g0 = P.row_group[m.lidx + r0], g1 = P.row_group[m.lidx + r1 - 1];
    for (int g = g0; g <= g1; ++g) arrivals[P.groups[g].t]++;
  };
  auto signal_all_tiles = [&](int s) {
    const SnMeta& m = P.meta[s];
    for (int r0 = m.w; r0 < m.h; r0 += 64) signal_rows(s, r0, std::min(m.h, r0 + 64));
  };
  for (const SolveTask& t : P.fwd_tasks) {
    if (t.kind == 6) {
      for (int j = t.i; j < t.i + t.t; ++j) signal_all_tiles(P.tiny[j]);
    } else if (t.kind == 4) {
      signal_all_tiles(t.s);
    } else if (t.kind == 2) {
      const SnMeta& m = P.meta[t.s];
      const int r0 = m.w + 64 * t.t;
      signal_rows(t.s, r0, std::min(m.h, r0 + 64));
    }
  }
  for (int s = 0; s < P.nsuper; ++s)
    CHECK(arrivals[s] == P.fwd_pending[s], "%s: supernode %d gets %lld forward arrivals, waits for %d", what, s,
          (long long)arrivals[s], P.fwd_pending[s]);

  // both sweeps run one task at a time in dispatch order with the kernels' wait targets and
  // signals (solve.cu): no task ever waits, and every supernode ends done
  const int SB = P.solve_sb, TPT = P.solve_tpt;
  auto nblk_of = [&](int s) { return (P.meta[s].w + 63) / 64; };
  auto nsb_of = [&](int s) { return (nblk_of(s) + SB - 1) / SB; };
  auto nb_in = [&](int s, int p) { return std::min(SB, nblk_of(s) - p * SB); };
  for (int sweep = 0; sweep < 2; ++sweep) {
    std::vector<int64_t> arrived(P.nsuper, 0), done(P.nsuper, 0), upd(std::max(1, P.nsb_total), 0);
    const std::vector<SolveTask>& tasks = sweep == 0 ? P.fwd_tasks : P.bwd_tasks;
    auto need = [&](bool ok, size_t i, const char* which) {
      CHECK(ok, "%s: %s task %zu (%s) would wait for a task handed out after it", what,
            sweep ? "backward" : "forward", i, which);
    };
    auto parent_done = [&](int s) {
      const int par = P.sparent[s];
      return par < 0 || done[par] >= solve_done_count(P.meta[par].w, SB, TPT);
    };
    for (size_t i = 0; i < tasks.size(); ++i) {
      const SolveTask& t = tasks[i];
      const int s = t.s;
      const SnMeta& m = P.meta[s];
      const int p = t.i & 0xffffff, nblk = nblk_of(s), nsb = nsb_of(s), noff = (m.h - m.w + 63) / 64;
      if (sweep == 0) {
        switch (t.kind) {
          case 6:
            for (int j = t.i; j < t.i + t.t; ++j) {
              const int q = P.tiny[j];
              for (int r0 = P.meta[q].w; r0 < P.meta[q].h; r0 += 64) {
                const int g0 = P.row_group[P.meta[q].lidx + r0];
                const int g1 = P.row_group[P.meta[q].lidx + std::min(P.meta[q].h, r0 + 64) - 1];
                for (int g = g0; g <= g1; ++g) arrived[P.groups[g].t]++;
              }
              done[q]++;
            }
            break;
          case 5:
            need(arrived[s] >= P.fwd_pending[s] && upd[m.sboff + p] >= (int64_t)p * nb_in(s, p) * solve_ntask(SB, TPT),
                 i, "DI");
            done[s]++;
            break;
          case 1:
            need(done[s] >= solve_di_range(nblk, SB, TPT, 0, p + 1), i, "U");
            upd[m.sboff + t.t / SB]++;
            break;
          case 2: {
            need(nblk == 1 ? done[s] >= 1 : done[s] >= solve_di_range(nblk, SB, TPT, 0, p + 1), i, "O");
            const int r0 = m.w + 64 * t.t, g0 = P.row_group[m.lidx + r0];
            const int g1 = P.row_group[m.lidx + std::min(m.h, r0 + 64) - 1];
            for (int g = g0; g <= g1; ++g) arrived[P.groups[g].t]++;
            break;
          }
          case 0:
            need(arrived[s] >= P.fwd_pending[s], i, "D");
            done[s]++;
            break;
          case 4:
            need(arrived[s] >= P.fwd_pending[s], i, "F");
            for (int r0 = m.w; r0 < m.h; r0 += 64) {
              const int g0 = P.row_group[m.lidx + r0], g1 = P.row_group[m.lidx + std::min(m.h, r0 + 64) - 1];
              for (int g = g0; g <= g1; ++g) arrived[P.groups[g].t]++;
            }
            done[s]++;
            break;
          default:
            CHECK(false, "%s: unknown forward task kind %d", what, t.kind);
        }
      } else {
        switch (t.kind) {
          case 6:
            for (int j = t.i; j < t.i + t.t; ++j) {
              need(parent_done(P.tiny[j]), i, "T");
              done[P.tiny[j]]++;
            }
            break;
          case 5: {
            const int nlast = nblk - (nsb - 1) * SB;
            const int later = p < nsb - 1 ? (nsb - 2 - p) * solve_ntask(SB, TPT) + solve_ntask(nlast, TPT) : 0;
            need(upd[m.sboff + p] >= (int64_t)noff * solve_ntask(nb_in(s, p), TPT) + (int64_t)nb_in(s, p) * later, i,
                 "DI");
            done[s]++;
            break;
          }
          case 1:
            need(done[s] >= solve_di_range(nblk, SB, TPT, p, nsb), i, "V");
            upd[m.sboff + t.t / SB]++;
            break;
          case 3:
            need(parent_done(s), i, "W");
            upd[m.sboff + p]++;
            break;
          case 0:
            need(upd[m.sboff] >= noff, i, "B");
            done[s]++;
            break;
          case 4:
            need(parent_done(s), i, "G");
            done[s]++;
            break;
          default:
            CHECK(false, "%s: unknown backward task kind %d", what, t.kind);
        }
      }
    }
    for (int s = 0; s < P.nsuper; ++s)
      CHECK(done[s] == solve_done_count(P.meta[s].w, SB, TPT), "%s: %s sweep leaves supernode %d at %lld of %d",
            what, sweep ? "backward" : "forward", s, (long long)done[s], solve_done_count(P.meta[s].w, SB, TPT));
  }
  for (int s = 0; s < P.nsuper; ++s) {
    const bool tiny = seen[s] > 0;
    CHECK(tiny == (fwd_tasks_of[s] == 0), "%s: supernode %d forward tasks %d tiny %d", what, s, fwd_tasks_of[s], tiny);
    CHECK(tiny == (bwd_tasks_of[s] == 0), "%s: supernode %d backward tasks %d tiny %d", what, s, bwd_tasks_of[s], tiny);
    if (tiny) CHECK(P.fwd_pending[s] == 0, "%s: tiny supernode %d expects arrivals", what, s);
  }
}

int main() {
  for (int full = 0; full < 2; ++full)
    for (int k : {6, 12, 20, 28}) {
      std::vector<int64_t> cp;
      std::vector<int32_t> ri;
      grid_matrix(k, full, cp, ri);
      const int n = k * k * k;
      const Symbolic sym = symbolic_factorization(n, cp.data(), ri.data(), OrderingKind::MMD, RelaxParams());
      char what[64];
      PlanParams p64;
      p64.factor_dag = true;
      std::snprintf(what, sizeof what, "%s %d^3 FP64", full ? "27-point" : "7-point", k);
      check_plan(sym, p64, what);
      PlanParams p32;
      p32.fp32 = true;
      p32.factor_dag = true;
      std::snprintf(what, sizeof what, "%s %d^3 FP32", full ? "27-point" : "7-point", k);
      check_plan(sym, p32, what);
      PlanParams small;
      small.factor_dag = true;
      small.outer_nb = 64;
      small.big_tile_rows = 96;
      small.small_max_w = 16;
      small.solve_sb = 3;
      small.solve_tpt = 1;
      std::snprintf(what, sizeof what, "%s %d^3 FP64 small blocks", full ? "27-point" : "7-point", k);
      check_plan(sym, small, what);
    }
  // a plan large enough (over 2^20 relative indices) for its relative indices to be
  // filled by several host threads
  {
    std::vector<int64_t> cp;
    std::vector<int32_t> ri;
    grid_matrix(44, true, cp, ri);
    const Symbolic sym = symbolic_factorization(44 * 44 * 44, cp.data(), ri.data(), OrderingKind::MMD, RelaxParams());
    const long long before = n_rel;
    check_plan(sym, PlanParams(), "27-point 44^3 FP64");
    CHECK(n_rel - before > (1 << 20), "27-point 44^3: only %lld relative indices", n_rel - before);
    // the assembly map (filled by host threads above 2^20 entries): every entry of A lands
    // on its (row, column) of the permuted factor inside its supernode's panel
    PlanParams np;
    np.factor_dag = false;
    const Plan P = build_plan(sym, np);
    const std::vector<int64_t> amap = build_assembly_map(sym, P, cp.data(), ri.data());
    CHECK((int64_t)amap.size() == cp.back() - 1 && amap.size() > (1u << 20), "assembly map size %zu", amap.size());
    bool bad = false;
    for (int c = 1; c <= sym.n && !bad; ++c)
      for (int64_t p = cp[c - 1]; p < cp[c] && !bad; ++p) {
        int pr = sym.invp[ri[p - 1] - 1] - 1, pc = sym.invp[c - 1] - 1;
        if (pr < pc) std::swap(pr, pc);
        const SnMeta& m = P.meta[P.supmember0[pc]];
        const int64_t d = amap[p - 1] - m.off, col = d / m.ld, pos = d % m.ld;
        bad = d < 0 || col != pc - m.fc || pos >= m.h || P.rows[m.lidx + pos] != pr;
      }
    CHECK(!bad, "27-point 44^3: an assembly map entry is not its (row, column) in the panel");
  }
  // a block-diagonal batch (a forest of elimination trees, merged as the batch analysis
  // merges its systems): grids, a dense block wider than one outer block, a path, and
  // many one-column systems
  {
    std::vector<Symbolic> parts;
    std::vector<int64_t> cp;
    std::vector<int32_t> ri;
    auto add = [&](int n) {
      parts.push_back(symbolic_factorization(n, cp.data(), ri.data(), OrderingKind::MMD, RelaxParams()));
    };
    grid_matrix(9, true, cp, ri);
    add(9 * 9 * 9);
    dense_matrix(300, cp, ri);
    add(300);
    for (int k : {3, 5, 7}) {
      grid_matrix(k, false, cp, ri);
      add(k * k * k);
    }
    path_matrix(500, cp, ri);
    add(500);
    dense_matrix(1, cp, ri);
    for (int j = 0; j < 40; ++j) add(1);
    grid_matrix(14, false, cp, ri);
    add(14 * 14 * 14);
    const Symbolic forest = merge_symbolic(parts);
    PlanParams p64;
    p64.factor_dag = true;
    check_plan(forest, p64, "batch FP64");
    PlanParams p32;
    p32.fp32 = true;
    p32.factor_dag = true;
    check_plan(forest, p32, "batch FP32");
    PlanParams small;
    small.factor_dag = true;
    small.outer_nb = 64;
    small.big_tile_rows = 96;
    small.small_max_w = 16;
    small.solve_sb = 3;
    small.solve_tpt = 1;
    check_plan(forest, small, "batch FP64 small blocks");
  }
  if (fails) {
    std::fprintf(stderr, "%d violations\n", fails);
    return 1;
  }
  std::printf("ok: %lld tiles (%lld tensor-core), %lld factor tasks, %lld tiny leaves, %lld relative indices\n",
              n_tiles, n_big_tiles, n_ftasks, n_tiny, n_rel);
  return 0;
}
