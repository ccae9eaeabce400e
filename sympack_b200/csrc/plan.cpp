#include "plan.hpp"

#include <algorithm>
#include <atomic>
#include <queue>
#include <stdexcept>
#include <system_error>
#include <thread>
#include <utility>

namespace spb {

static int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

static void build_factor_dag(Plan& P, const PlanParams& prm, const std::vector<double>* measured_us = nullptr);

Plan build_plan(const Symbolic& sym, const PlanParams& prm) {
  Plan P;
  P.n = sym.n;
  P.nsuper = sym.nsuper();
  const int ns = P.nsuper;
  P.meta.resize(ns);
  P.rows.resize(sym.lindx.size());
  for (size_t k = 0; k < sym.lindx.size(); ++k) P.rows[k] = sym.lindx[k] - 1;
  P.lindx_total = (int64_t)sym.lindx.size();
  P.supmember0.resize(sym.n);
  for (int i = 0; i < sym.n; ++i) P.supmember0[i] = sym.supmember[i] - 1;

  int64_t off = 0;
  for (int s = 0; s < ns; ++s) {
    SnMeta& m = P.meta[s];
    m.fc = sym.xsuper[s] - 1;
    m.w = sym.xsuper[s + 1] - sym.xsuper[s];
    m.h = (int32_t)(sym.xlindx[s + 1] - sym.xlindx[s]);
    m.ld = (int32_t)round_up(m.h, 4);
    m.off = off;
    m.lidx = sym.xlindx[s] - 1;
    m.boff = P.nblk_total;
    m.sboff = 0;
    m.ioff = -1;
    P.nblk_total += (m.w + 63) / 64;
    off += round_up((int64_t)m.ld * m.w, 32);
  }
  P.arena_elems = off;

  // supernodal elimination tree and height levels
  P.sparent.assign(ns, -1);
  for (int s = 0; s < ns; ++s) {
    int lc = sym.xsuper[s + 1] - 1;  // 1-based last column
    int pc = sym.parent[lc - 1];
    P.sparent[s] = pc ? sym.supmember[pc - 1] - 1 : -1;
  }
  P.level.assign(ns, 0);
  for (int s = 0; s < ns; ++s)  // children precede parents in postorder
    if (P.sparent[s] >= 0) P.level[P.sparent[s]] = std::max(P.level[P.sparent[s]], P.level[s] + 1);
  int H = 0;
  for (int s = 0; s < ns; ++s) H = std::max(H, P.level[s] + 1);
  P.nlevels = H;
  P.level_sn.assign(H, {});
  for (int s = 0; s < ns; ++s) P.level_sn[P.level[s]].push_back(s);

  P.is_big.assign(ns, 0);
  for (int s = 0; s < ns; ++s) {
    const SnMeta& m = P.meta[s];
    bool small = m.w <= prm.small_max_w && (int64_t)m.h * m.w * 8 <= prm.small_max_bytes;
    P.is_big[s] = small ? 0 : 1;
    double w = m.w, mm = m.h - m.w;
    P.exec_flops += w * w * w / 3.0 + mm * w * w + mm * mm * w;
  }

  // Tiles of a (rend-rbeg) x (cend-cbeg) product, rows/cols counted from rbeg/cbeg;
  // tiles entirely above the diagonal of a symmetric product are skipped.
  // FP64 tensor-core tiles are 128 x 64 and copy their operands' columns from the even row
  // at or below their first row, so they are cut from even rows (the first tile of a range
  // that starts on an odd row has one row fewer).
  auto push_tiles = [&](std::vector<TileItem>& out, int T, int s, int mode, int rbeg, int rend, int cbeg, int cend,
                        int k0, int kn) {
    const bool dmma = T == 128 && !prm.fp32;
    const int TN = dmma ? 64 : T;
    const int r00 = dmma ? (rbeg & ~1) : rbeg, c00 = dmma ? (cbeg & ~1) : cbeg;
    for (int cj = c00; cj < cend; cj += TN)
      for (int ri = r00; ri < rend; ri += T) {
        if (ri + T <= cj) continue;  // rows and columns are both panel rows: tile above the diagonal
        TileItem t;
        t.s = s;
        t.mode = mode;
        t.a_row0 = std::max(ri, rbeg);
        t.b_row0 = std::max(cj, cbeg);
        t.k0 = k0;
        t.kn = kn;
        t.mrows = std::min(ri + T, rend) - t.a_row0;
        t.ncols = std::min(cj + TN, cend) - t.b_row0;
        out.push_back(t);
      }
  };
  // A launch with fewer tiles than the GPU has slots for them splits each tile's K range
  // into parts of at least 64 columns (split-K): the update epilogue subtracts with
  // atomic additions, so the partial products of one tile simply add up.
  auto split_k = [&](std::vector<TileItem>& v, int per_sm) {
    const int64_t slots = (int64_t)std::max(1, prm.sms) * per_sm;
    if (v.empty() || (int64_t)v.size() * 2 > slots) return;
    const int parts = (int)std::min<int64_t>(8, slots / (int64_t)v.size());  // one wave
    std::vector<TileItem> out;
    out.reserve(v.size() * parts);
    for (const TileItem& t : v) {
      const int p = std::min(parts, t.kn / 64);
      if (p <= 1) {
        out.push_back(t);
        continue;
      }
      const int step = (t.kn / p + 63) / 64 * 64;
      for (int k = 0; k < t.kn; k += step) {
        TileItem u = t;
        u.k0 = t.k0 + k;
        u.kn = std::min(step, t.kn - k);
        out.push_back(u);
      }
    }
    v.swap(out);
  };
  // Emit the tiles of one phase as (up to) two launches: 64-wide FMA tiles and
  // 128-wide tensor-core tiles.
  std::vector<TileItem> t64, t128;
  auto flush_gemm = [&](Lane lane, int blk) {
    for (int pass = 0; pass < 2; ++pass) {
      std::vector<TileItem>& v = pass ? t128 : t64;
      if (v.empty()) continue;
      split_k(v, pass ? (prm.fp32 ? 1 : 2) : 4);  // CTAs per SM of the tile engines
      Step gs{StepKind::Gemm, (int32_t)P.tile_items.size(), (int32_t)v.size(), 0, pass ? 128 : 64, lane, blk};
      P.tile_items.insert(P.tile_items.end(), v.begin(), v.end());
      P.steps.push_back(gs);
      v.clear();
    }
  };
  auto pick = [&](int rows) -> std::vector<TileItem>& { return rows >= prm.big_tile_rows ? t128 : t64; };
  auto tile_of = [&](int rows) { return rows >= prm.big_tile_rows ? 128 : 64; };

  for (int L = 0; L < H; ++L) {
    const auto& sns = P.level_sn[L];
    // 1. fused small panels
    {
      Step st{StepKind::FactorSmall, (int32_t)P.small_items.size(), 0, 0, 0};
      st.lane = Lane::Join;
      for (int s : sns)
        if (!P.is_big[s]) {
          P.small_items.push_back(s);
          st.arg = std::max<int32_t>(st.arg, P.meta[s].h * P.meta[s].w * 8);
        }
      st.count = (int32_t)P.small_items.size() - st.begin;
      if (st.count) P.steps.push_back(st);
    }
    // 2. blocked factorization of big panels, all big panels of the level in lockstep
    int maxw = 0;
    for (int s : sns)
      if (P.is_big[s]) maxw = std::max(maxw, P.meta[s].w);
    const int outer = std::max(prm.nb, prm.outer_nb / prm.nb * prm.nb);
    for (int c0 = 0; c0 < maxw; c0 += prm.nb) {
      const int blk = c0 / prm.nb;
      Step pd{StepKind::PotrfDiag, (int32_t)P.panel_items.size(), 0, c0, 0, Lane::Chain, blk};
      // every diagonal block has its own scratch slot (the persistent factorization keeps
      // several blocks of one supernode in flight)
      const int slot0 = P.max_diag_slots;
      int nslots = 0;
      for (int s : sns) {
        if (!P.is_big[s] || c0 >= P.meta[s].w) continue;
        P.panel_items.push_back(PanelItem{s, c0, std::min(prm.nb, P.meta[s].w - c0), -1, slot0 + nslots++});
      }
      P.max_diag_slots = slot0 + nslots;
      pd.count = (int32_t)P.panel_items.size() - pd.begin;
      if (pd.count) P.steps.push_back(pd);
      Step pt{StepKind::TrsmRows, (int32_t)P.panel_items.size(), 0, c0, 0, Lane::Chain, blk};
      int slot = 0;
      for (int s : sns) {
        if (!P.is_big[s]) continue;
        const SnMeta& m = P.meta[s];
        if (c0 >= m.w) continue;
        int nbk = std::min(prm.nb, m.w - c0);
        for (int r = c0 + nbk; r < m.h; r += 64) P.panel_items.push_back(PanelItem{s, c0, nbk, r, slot0 + slot});
        ++slot;
      }
      pt.count = (int32_t)P.panel_items.size() - pt.begin;
      if (pt.count) P.steps.push_back(pt);
      // update inside the outer block (columns up to its end) with this block, on the chain
      for (int s : sns) {
        if (!P.is_big[s]) continue;
        const SnMeta& m = P.meta[s];
        if (c0 >= m.w) continue;
        const int nbk = std::min(prm.nb, m.w - c0), c1 = c0 + nbk;
        const int oend = std::min(m.w, (c0 / outer + 1) * outer);
        if (c1 >= oend) continue;
        const int rows = m.h - c1;
        push_tiles(pick(rows), tile_of(rows), s, 0, c1, m.h, c1, oend, c0, nbk);
      }
      flush_gemm(Lane::Chain, blk);
      // end of an outer block: update every later column with the whole outer block
      // (K = outer width); the first column tile (it holds the next block) on the
      // chain, the remaining columns on the side lane
      if ((c0 + prm.nb) % outer == 0 || c0 + prm.nb >= maxw) {
        const int ob = c0 / outer * outer;
        for (int pass = 0; pass < 2; ++pass) {
          for (int s : sns) {
            if (!P.is_big[s]) continue;
            const SnMeta& m = P.meta[s];
            if (ob >= m.w) continue;
            const int oe = std::min(m.w, ob + outer);
            if (oe >= m.w || c0 + prm.nb < oe) continue;  // a narrower panel ended its outer block earlier
            const int rows = m.h - oe, T = tile_of(rows);
            if (pass == 0) push_tiles(pick(rows), T, s, 0, oe, m.h, oe, std::min(m.w, oe + T), ob, oe - ob);
            else if (oe + T < m.w) push_tiles(pick(rows), T, s, 0, oe, m.h, oe + T, m.w, ob, oe - ob);
          }
          flush_gemm(pass == 0 ? Lane::Chain : Lane::Side, blk);
        }
      }
    }
    // 3. external Schur-complement updates of every panel of the level
    for (int s : sns) {
      const SnMeta& m = P.meta[s];
      int rows = m.h - m.w;
      if (rows > 0) push_tiles(pick(rows), tile_of(rows), s, 1, m.w, m.h, m.w, m.h, 0, m.w);
    }
    flush_gemm(Lane::Join, 0);
  }
  // relative indices of the external updates: groups of off-diagonal rows by target
  // (every row of s from a group's first one on is in its target's row list), the
  // group's positions in the target found by merging the sorted row lists from the
  // first row's place.  The groups and their offsets first, then the positions,
  // groups spread over host threads (batches of many systems have 1e8+ positions).
  P.row_group.assign(P.rows.size(), -1);
  int64_t nrel = 0;
  std::vector<int32_t> group_s;  // source supernode of each group
  for (int s = 0; s < ns; ++s) {
    const SnMeta& m = P.meta[s];
    const int32_t* rl = P.rows.data() + m.lidx;
    int r = m.w;
    while (r < m.h) {
      const int t = P.supmember0[rl[r]];
      const int gid = (int)P.groups.size();
      P.groups.push_back(RelGroup{t, r, nrel});
      group_s.push_back(s);
      nrel += m.h - r;
      int e = r;
      while (e < m.h && P.supmember0[rl[e]] == t) P.row_group[m.lidx + e++] = gid;
      r = e;
    }
  }
  P.rel.resize((size_t)nrel);
  {
    std::atomic<int64_t> next{0};
    std::atomic<bool> missing{false};
    const int64_t ngroups = (int64_t)P.groups.size(), chunk = 256;
    auto fill = [&]() {
      for (int64_t g0 = next.fetch_add(chunk); g0 < ngroups; g0 = next.fetch_add(chunk)) {
        for (int64_t g = g0; g < std::min(ngroups, g0 + chunk); ++g) {
          const RelGroup& gr = P.groups[g];
          const SnMeta& m = P.meta[group_s[g]];
          const SnMeta& mt = P.meta[gr.t];
          const int32_t* rl = P.rows.data() + m.lidx;
          const int32_t* tl = P.rows.data() + mt.lidx;
          int32_t* out = P.rel.data() + gr.rel_off;
          int q = (int)(std::lower_bound(tl, tl + mt.h, rl[gr.j0]) - tl);
          for (int i = gr.j0; i < m.h; ++i) {
            while (q < mt.h && tl[q] < rl[i]) ++q;
            if (q == mt.h || tl[q] != rl[i]) {
              missing = true;
              return;
            }
            out[i - gr.j0] = q;
          }
        }
      }
    };
    const unsigned nth = nrel < (1 << 20) ? 1u : std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    try {
      for (unsigned k = 1; k < nth; ++k) pool.emplace_back(fill);
    } catch (const std::system_error&) {  // fewer threads: the ones started and this one share the groups
    }
    fill();
    for (std::thread& th : pool) th.join();
    if (missing) throw std::runtime_error("plan: update row missing from its target's structure");
  }

  // algorithmic flops per step
  P.step_flops.assign(P.steps.size(), 0.0);
  for (size_t k = 0; k < P.steps.size(); ++k) {
    const Step& st = P.steps[k];
    double f = 0.0;
    for (int i = st.begin; i < st.begin + st.count; ++i) {
      if (st.kind == StepKind::FactorSmall) {
        const SnMeta& m = P.meta[P.small_items[i]];
        double w = m.w, mm = m.h - m.w;
        f += w * w * w / 3.0 + mm * w * w;
      } else if (st.kind == StepKind::PotrfDiag) {
        double nb = P.panel_items[i].nb;
        f += nb * nb * nb / 3.0;
      } else if (st.kind == StepKind::TrsmRows) {
        const PanelItem& it = P.panel_items[i];
        double rows = std::min(64, P.meta[it.s].h - it.row0);
        f += rows * it.nb * it.nb;
      } else {
        const TileItem& t = P.tile_items[i];
        // pairs (r, c) of the tile with panel row >= panel column: column c (panel row
        // b_row0 + c) pairs with the tile rows from max(0, d + c) on, d = b_row0 - a_row0
        const int64_t d = t.b_row0 - t.a_row0, mr = t.mrows, nc = t.ncols;
        const int64_t c0 = std::min(nc, std::max<int64_t>(0, 1 - d));  // columns paired with every row
        const int64_t k = std::max<int64_t>(0, std::min(nc, mr - d) - c0);  // then mr - d - c rows each
        const int64_t pairs = c0 * mr + k * (mr - d) - (k * c0 + k * (k - 1) / 2);
        f += 2.0 * t.kn * (double)pairs;
      }
    }
    P.step_flops[k] = f;
  }
  for (const SnMeta& m : P.meta) P.solve_sweep_bytes += 8.0 * m.h * m.w;
  if (prm.factor_dag) build_factor_dag(P, prm);

  // Solve super-blocks: per supernode, its first super-block counter and (for
  // supernodes wider than one block) the offset of its inverse tiles.
  const int SB = std::max(1, prm.solve_sb);
  const int TPT = std::max(1, prm.solve_tpt);
  P.solve_sb = SB;
  P.solve_tpt = TPT;
  auto nblk_of = [&](int s) { return (P.meta[s].w + 63) / 64; };
  auto nsb_of = [&](int s) { return (nblk_of(s) + SB - 1) / SB; };
  auto nb_in = [&](int s, int p) { return std::min(SB, nblk_of(s) - p * SB); };
  for (int s = 0; s < ns; ++s) {
    SnMeta& m = P.meta[s];
    m.sboff = P.nsb_total;
    P.nsb_total += nsb_of(s);
    if (nblk_of(s) > 1) {
      m.ioff = P.inv_elems;
      for (int p = 0; p < nsb_of(s); ++p) {
        P.inv_elems += inv_tiles(nb_in(s, p)) * 4096;
        for (int j = 0; j < nb_in(s, p); ++j) P.inv_items.push_back(InvItem{s, p, j, 0});
      }
    }
  }
  // Longest inverse items first (column block 0 of a full super-block has the most tiles).
  std::stable_sort(P.inv_items.begin(), P.inv_items.end(), [&](const InvItem& x, const InvItem& y) {
    return nb_in(x.s, x.p) - x.j > nb_in(y.s, y.p) - y.j;
  });

  // Persistent solve task lists, ordered by elimination-tree height level
  // (forward: leaves first; backward: root level first) so that tasks handed
  // out together are independent.  The supernodes of a level advance together:
  // tasks are dealt super-block by super-block across the level, so sibling
  // supernodes run side by side.  Within a super-block the tasks on the critical
  // path come first: the DI tasks, then the updates of the next super-block, then
  // the other updates and the off-diagonal tiles.  A task covers up to TPT tiles.
  auto chunks = [&](std::vector<SolveTask>& out, int s, int kind, int p, int t, int q_begin, int q_end) {
    for (int q0 = q_begin; q0 < q_end; q0 += TPT) out.push_back(SolveTask{s, kind, pack_task_i(p, q0 - q_begin), t});
  };
  P.fwd_pending.assign(ns, 0);
  // tiny leaves first: a thread each, no waits
  auto tiny_leaf = [&](int s) {
    const SnMeta& m = P.meta[s];
    return P.level[s] == 0 && m.w <= kTinyMaxW && (int64_t)m.w * m.h <= kTinyMaxElems;
  };
  P.tiny.clear();
  if (H > 0)
    for (int s : P.level_sn[0])
      if (tiny_leaf(s)) P.tiny.push_back(s);
  for (size_t i = 0; i < P.tiny.size(); i += kTinyBatch)
    P.fwd_tasks.push_back(SolveTask{P.tiny[i], 6, (int32_t)i,
                                    (int32_t)std::min<size_t>(kTinyBatch, P.tiny.size() - i)});
  for (int L = 0; L < H; ++L) {
    int maxsb = 0;
    for (int s : P.level_sn[L]) maxsb = std::max(maxsb, nsb_of(s));
    for (int p = 0; p < maxsb; ++p)
      for (int s : P.level_sn[L]) {
        const SnMeta& m = P.meta[s];
        const int nblk = nblk_of(s), noff = (m.h - m.w + 63) / 64;
        if (p >= nsb_of(s)) continue;
        if (tiny_leaf(s)) continue;
        if (nblk == 1) {
          if (noff <= kSolveFusedTiles) {  // the whole supernode in one task
            P.fwd_tasks.push_back(SolveTask{s, 4, 0, 0});
          } else {
            P.fwd_tasks.push_back(SolveTask{s, 0, 0, 0});
            for (int u = 0; u < noff; ++u) P.fwd_tasks.push_back(SolveTask{s, 2, 0, u});
          }
          continue;
        }
        const int nb = nb_in(s, p);
        for (int r = 0; r < nb; ++r) chunks(P.fwd_tasks, s, 5, p, r, 0, r + 1);
        for (int t = (p + 1) * SB; t < nblk; ++t) chunks(P.fwd_tasks, s, 1, p, t, 0, nb);
        for (int u = 0; u < noff; ++u) chunks(P.fwd_tasks, s, 2, p, u, 0, nb);
      }
    // arrivals: one per (off-diagonal task, target supernode of its tile)
    for (int s : P.level_sn[L]) {
      const SnMeta& m = P.meta[s];
      const int noff = (m.h - m.w + 63) / 64;
      int nsrc = 0;
      for (int p = 0; p < nsb_of(s); ++p) nsrc += solve_ntask(nb_in(s, p), TPT);
      for (int u = 0; u < noff; ++u) {
        int r0 = m.w + 64 * u, r1 = std::min(m.h, r0 + 64), last = -1;
        for (int r = r0; r < r1; ++r) {
          int t = P.supmember0[P.rows[m.lidx + r]];
          if (t != last) P.fwd_pending[t] += nsrc;
          last = t;
        }
      }
    }
  }
  for (int L = H - 1; L >= 0; --L) {
    int maxsb = 0;
    for (int s : P.level_sn[L]) maxsb = std::max(maxsb, nsb_of(s));
    for (int j = 0; j < maxsb; ++j)
      for (int s : P.level_sn[L]) {
        const SnMeta& m = P.meta[s];
        const int nblk = nblk_of(s), noff = (m.h - m.w + 63) / 64, nsb = nsb_of(s);
        if (j >= nsb) continue;
        if (tiny_leaf(s)) continue;
        if (nblk == 1) {
          if (noff <= kSolveFusedTiles) {
            P.bwd_tasks.push_back(SolveTask{s, 4, 0, 0});
          } else {
            for (int u = 0; u < noff; ++u) P.bwd_tasks.push_back(SolveTask{s, 3, 0, u});
            P.bwd_tasks.push_back(SolveTask{s, 0, 0, 0});
          }
          continue;
        }
        const int p = nsb - 1 - j, nb = nb_in(s, p);  // super-blocks from the last one down
        for (int u = 0; u < noff; ++u) chunks(P.bwd_tasks, s, 3, p, u, 0, nb);
        for (int r = nb - 1; r >= 0; --r) chunks(P.bwd_tasks, s, 5, p, r, 0, nb - r);
        for (int t = p * SB - 1; t >= 0; --t) chunks(P.bwd_tasks, s, 1, p, t, 0, nb);
      }
  }
  for (size_t i = 0; i < P.tiny.size(); i += kTinyBatch)  // the tiny leaves last
    P.bwd_tasks.push_back(SolveTask{P.tiny[i], 6, (int32_t)i,
                                    (int32_t)std::min<size_t>(kTinyBatch, P.tiny.size() - i)});
  return P;
}

std::vector<int64_t> build_assembly_map(const Symbolic& sym, const Plan& P, const int64_t* colptr,
                                        const int32_t* rowind) {
  const int n = sym.n;
  const int64_t nnz = colptr[n] - 1;
  std::vector<int64_t> dst(nnz);
  std::atomic<int> next{1};
  std::atomic<bool> outside{false};
  const int chunk = 4096;
  auto fill = [&]() {  // columns in chunks; every entry's place is independent of the others
    for (int c0 = next.fetch_add(chunk); c0 <= n; c0 = next.fetch_add(chunk)) {
      for (int c = c0; c < std::min(n + 1, c0 + chunk); ++c)
        for (int64_t p = colptr[c - 1]; p < colptr[c]; ++p) {
          int r = rowind[p - 1];
          int pr = sym.invp[r - 1] - 1, pc = sym.invp[c - 1] - 1;
          if (pr < pc) std::swap(pr, pc);
          int s = P.supmember0[pc];
          const SnMeta& m = P.meta[s];
          const int32_t* rl = P.rows.data() + m.lidx;
          const int32_t* it = std::lower_bound(rl, rl + m.h, pr);
          if (it == rl + m.h || *it != pr) {
            outside = true;
            return;
          }
          dst[p - 1] = m.off + (int64_t)(pc - m.fc) * m.ld + (it - rl);
        }
    }
  };
  const unsigned nth = nnz < (1 << 20) ? 1u : std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  try {
    for (unsigned k = 1; k < nth; ++k) pool.emplace_back(fill);
  } catch (const std::system_error&) {  // fewer threads: the ones started and this one share the columns
  }
  fill();
  for (std::thread& th : pool) th.join();
  if (outside) throw std::runtime_error("assembly: entry outside the symbolic structure");
  return dst;
}

// Persistent factorization: the items of the step sequence as one task graph.
//   small panel s        waits ext[s] complete                        bumps sdone[s]
//   POTRF of block b     waits ext[s] complete and col[b] complete    bumps blk[b], sdone[s]
//   TRSM row tile of b   waits blk[b] >= 1 (its POTRF)                bumps blk[b], sdone[s]
//   in-panel update      waits blk[b] complete for its K blocks       bumps col[c] of its column blocks
//   external update      waits sdone[s] complete                      bumps ext[t] of its targets
// (the reference's FACTOR -> TRSM -> UPDATE dependencies, symPACKMatrix2D.hpp:3893-3997, at
// block granularity).  The dispatch order comes from a list-scheduling simulation on
// the SMs with estimated task times, highest bottom level first, and is topological:
// a CTA only ever waits for tasks handed out before its own.
void reorder_factor_tasks(Plan& P, const PlanParams& prm, const std::vector<double>& us) {
  if (us.size() != P.ftasks.size()) throw std::invalid_argument("reorder: one duration per factor task");
  build_factor_dag(P, prm, &us);
}

// measured_us: durations of the current tasks, in their dispatch order (P.ftasks), used in
// place of the cost model for the tasks they name.
static void build_factor_dag(Plan& P, const PlanParams& prm, const std::vector<double>* measured_us) {
  const int ns = P.nsuper, nb = P.nblk_total;
  const int EXT = 0, SDONE = ns, BLK = 2 * ns, COL = 2 * ns + nb;
  P.nfctr = 2 * ns + 2 * nb;
  std::vector<int32_t> e_ext(ns, 0), e_sdone(ns, 0), e_blk(nb, 0), e_col(nb, 0);
  struct Raw {
    int kind, item, s;
    int32_t nsig;
    int64_t sig0;  // signals sigv[sig0 .. sig0 + nsig)
    double us;
  };
  std::vector<Raw> raw;
  std::vector<int32_t> sigv;  // every task's signals, flat (millions of tasks in a batch)
  size_t ntask_all = 0;
  for (const Step& st : P.steps) ntask_all += (size_t)st.count;
  raw.reserve(ntask_all);
  sigv.reserve(ntask_all * 2);
  // tasks of each step in step order (already topological), signals first
  for (const Step& st : P.steps) {
    for (int i = st.begin; i < st.begin + st.count; ++i) {
      Raw r;
      r.item = i;
      r.sig0 = (int64_t)sigv.size();
      if (st.kind == StepKind::FactorSmall) {
        const int s = P.small_items[i];
        const SnMeta& m = P.meta[s];
        r.kind = 0;
        r.s = s;
        sigv.push_back(SDONE + s);
        const double w = m.w, mm = m.h - m.w;
        r.us = 2.2 + 13.0 * (w * w * w / 3.0 + mm * w * w) / 20e3;
        e_sdone[s] += 1;
      } else if (st.kind == StepKind::PotrfDiag || st.kind == StepKind::TrsmRows) {
        const PanelItem& it = P.panel_items[i];
        const int b = P.meta[it.s].boff + it.c0 / 64;
        r.kind = st.kind == StepKind::PotrfDiag ? 1 : 2;
        r.s = it.s;
        sigv.push_back(BLK + b);
        sigv.push_back(SDONE + it.s);
        r.us = r.kind == 1 ? 24.0 : 12.0;
        e_blk[b] += 1;
        e_sdone[it.s] += 1;
      } else {
        const TileItem& t = P.tile_items[i];
        const SnMeta& m = P.meta[t.s];
        r.kind = st.tile == 128 ? 4 : 3;
        r.s = t.s;
        const double fl = 2.0 * t.mrows * t.ncols * t.kn;
        // fixed cost + per-CTA rate (FP64 128 x 64 tiles at two CTAs per SM, FP32 3xTF32
        // tiles at one).  The FP64 figures, like the small-panel, diagonal-block and TRSM
        // times above, fit the per-kind duration quantiles of the task timeline of a traced
        // 60^3 Laplacian factorization (spb_get_factor_trace): a 128 x 64 tile costs about
        // 11 us before its first flop (pipeline fill, dependency reads, atomic epilogue)
        r.us = st.tile == 128 ? (prm.fp32 ? 3.0 + fl / 600e3 : 11.0 + fl / 105e3) : 5.0 + fl / 16.7e3;
        if (t.mode == 0) {
          for (int c = t.b_row0 / 64; c <= (t.b_row0 + t.ncols - 1) / 64; ++c) {
            sigv.push_back(COL + m.boff + c);
            e_col[m.boff + c] += 1;
          }
        } else {
          int last = -1;
          for (int c = 0; c < t.ncols; ++c) {
            const int g = P.row_group[m.lidx + t.b_row0 + c];
            const int tgt = P.groups[g].t;
            if (tgt != last) {
              sigv.push_back(EXT + tgt);
              e_ext[tgt] += 1;
            }
            last = tgt;
          }
        }
      }
      r.nsig = (int32_t)((int64_t)sigv.size() - r.sig0);
      raw.push_back(r);
    }
  }
  if (measured_us) {  // (kind, item) names a task: items index small_items, panel_items or tile_items
    std::vector<int32_t> of_small(P.small_items.size(), -1), of_panel(P.panel_items.size(), -1),
        of_tile(P.tile_items.size(), -1);
    for (size_t k = 0; k < raw.size(); ++k) {
      std::vector<int32_t>& of = raw[k].kind == 0 ? of_small : raw[k].kind <= 2 ? of_panel : of_tile;
      of[raw[k].item] = (int32_t)k;
    }
    for (size_t i = 0; i < P.ftasks.size(); ++i) {
      const FTask& t = P.ftasks[i];
      const std::vector<int32_t>& of = t.kind == 0 ? of_small : t.kind <= 2 ? of_panel : of_tile;
      const int32_t k = t.item >= 0 && t.item < (int32_t)of.size() ? of[t.item] : -1;
      if (k < 0 || raw[k].kind != t.kind) throw std::invalid_argument("reorder: tasks do not match the plan");
      const double d = (*measured_us)[i];
      if (d > 0.0 && d < 1e7) raw[k].us = d;  // else keep the model's estimate
    }
  }
  // waits of every task, flat: task k's are wv[woff[k] .. woff[k + 1])
  std::vector<FWait> wv;
  std::vector<int64_t> woff(raw.size() + 1, 0);
  wv.reserve(raw.size() * 2);
  for (size_t k = 0; k < raw.size(); ++k) {
    const Raw& r = raw[k];
    woff[k] = (int64_t)wv.size();
    if (r.kind == 0) {
      wv.push_back({EXT + r.s, e_ext[r.s]});
    } else if (r.kind == 1 || r.kind == 2) {
      const PanelItem& it = P.panel_items[r.item];
      const int b = P.meta[it.s].boff + it.c0 / 64;
      if (r.kind == 1) {
        wv.push_back({EXT + r.s, e_ext[r.s]});
        wv.push_back({COL + b, e_col[b]});
      } else {
        wv.push_back({BLK + b, 1});
      }
    } else {
      const TileItem& t = P.tile_items[r.item];
      const SnMeta& m = P.meta[t.s];
      if (t.mode == 0) {
        for (int c = t.k0 / 64; c <= (t.k0 + t.kn - 1) / 64; ++c) wv.push_back({BLK + m.boff + c, e_blk[m.boff + c]});
      } else {
        wv.push_back({SDONE + t.s, e_sdone[t.s]});
      }
    }
  }
  woff[raw.size()] = (int64_t)wv.size();
  // dependency graph for the simulation: every counter is a zero-time join node whose
  // predecessors are its signalling tasks; a task depends on the joins it waits for
  // (a TRSM tile waits for its block's POTRF only).  Successor lists in CSR form.
  const int nt = (int)raw.size(), nc = P.nfctr, nn = nt + nc;
  std::vector<int32_t> potrf_of(nb, -1);
  for (int k = 0; k < nt; ++k)
    if (raw[k].kind == 1) potrf_of[P.meta[P.panel_items[raw[k].item].s].boff + P.panel_items[raw[k].item].c0 / 64] = k;
  std::vector<int64_t> soff(nn + 1, 0);
  std::vector<int32_t> npred(nn, 0);
  auto for_edges = [&](auto&& edge) {
    for (int k = 0; k < nt; ++k) {
      for (int64_t q = raw[k].sig0; q < raw[k].sig0 + raw[k].nsig; ++q) edge(k, nt + sigv[q]);
      for (int64_t q = woff[k]; q < woff[k + 1]; ++q) {
        const FWait& w = wv[q];
        if (w.target <= 0) continue;
        edge(raw[k].kind == 2 ? potrf_of[w.ctr - BLK] : nt + w.ctr, k);
      }
    }
  };
  for_edges([&](int from, int to) {
    soff[from + 1]++;
    npred[to]++;
  });
  for (int v = 0; v < nn; ++v) soff[v + 1] += soff[v];
  std::vector<int32_t> sadj(soff[nn]);
  {
    std::vector<int64_t> fill(soff.begin(), soff.end() - 1);
    for_edges([&](int from, int to) { sadj[fill[from]++] = to; });
  }
  struct SuccRange {
    const int32_t* b;
    const int32_t* e;
    const int32_t* begin() const { return b; }
    const int32_t* end() const { return e; }
  };
  auto succ_of = [&](int v) { return SuccRange{sadj.data() + soff[v], sadj.data() + soff[v + 1]}; };
  // bottom levels (longest path to the end), in reverse topological order: counters
  // and tasks are processed after all their successors via a Kahn order
  std::vector<double> dur(nn, 0.0), blev(nn, 0.0);
  for (int k = 0; k < nt; ++k) dur[k] = raw[k].us;
  std::vector<int32_t> order;
  order.reserve(nn);
  {
    std::vector<int32_t> indeg = npred;
    for (int v = 0; v < nn; ++v)
      if (!indeg[v]) order.push_back(v);
    for (size_t q = 0; q < order.size(); ++q)
      for (int32_t u : succ_of(order[q]))
        if (--indeg[u] == 0) order.push_back(u);
    if ((int)order.size() != nn) throw std::runtime_error("plan: factorization task graph has a cycle");
  }
  for (int q = nn - 1; q >= 0; --q) {
    const int v = order[q];
    double best = 0.0;
    for (int32_t u : succ_of(v)) best = std::max(best, blev[u]);
    blev[v] = dur[v] + best;
  }
  // list scheduling on the SMs' CTA slots (two per SM for FP64, one for FP32)
  const int workers = std::max(1, prm.sms) * (prm.fp32 ? 1 : 2);
  std::vector<int32_t> pend = npred;
  // ready tasks by bottom level, ties to the lower index; the key travels with the task
  using Key = std::pair<double, int32_t>;
  auto cmp = [](const Key& x, const Key& y) { return x.first < y.first || (x.first == y.first && x.second > y.second); };
  std::priority_queue<Key, std::vector<Key>, decltype(cmp)> ready(cmp);
  using Ev = std::pair<double, int32_t>;
  std::priority_queue<Ev, std::vector<Ev>, std::greater<Ev>> running;
  std::vector<int32_t> dispatch;
  dispatch.reserve(nt);
  std::vector<int32_t> stack;
  auto complete = [&](int32_t v) {  // v finished: release successors, joins complete at once
    stack.push_back(v);
    while (!stack.empty()) {
      const int32_t x = stack.back();
      stack.pop_back();
      for (int32_t u : succ_of(x))
        if (--pend[u] == 0) {
          if (u >= nt) stack.push_back(u);
          else ready.push({blev[u], u});
        }
    }
  };
  for (int v = nt; v < nn; ++v)
    if (!pend[v]) complete(v);
  for (int v = 0; v < nt; ++v)
    if (!pend[v]) ready.push({blev[v], v});
  double now = 0.0;
  int busy = 0;
  while ((int)dispatch.size() < nt) {
    while (busy < workers && !ready.empty()) {
      const int32_t v = ready.top().second;
      ready.pop();
      dispatch.push_back(v);
      running.push({now + dur[v], v});
      ++busy;
    }
    if (running.empty()) throw std::runtime_error("plan: factorization schedule stalled");
    const Ev e = running.top();
    running.pop();
    now = e.first;
    --busy;
    complete(e.second);
  }
  while (!running.empty()) {
    now = running.top().first;
    running.pop();
  }
  P.fsim_us = now;
  P.ftasks.clear();
  P.fwaits.clear();
  P.fsigs.clear();
  P.ftasks.reserve(dispatch.size());
  P.fwaits.reserve(wv.size());
  P.fsigs.reserve(sigv.size());
  for (int32_t k : dispatch) {
    FTask t;
    t.kind = raw[k].kind;
    t.item = raw[k].item;
    t.wait0 = (int32_t)P.fwaits.size();
    for (int64_t q = woff[k]; q < woff[k + 1]; ++q)
      if (wv[q].target > 0) P.fwaits.push_back(wv[q]);
    t.nwait = (int32_t)P.fwaits.size() - t.wait0;
    t.w0_ctr = t.nwait > 0 ? P.fwaits[t.wait0].ctr : 0;
    t.w0_target = t.nwait > 0 ? P.fwaits[t.wait0].target : 0;
    t.sig0 = (int32_t)P.fsigs.size();
    P.fsigs.insert(P.fsigs.end(), sigv.begin() + raw[k].sig0, sigv.begin() + raw[k].sig0 + raw[k].nsig);
    t.nsig = raw[k].nsig;
    P.ftasks.push_back(t);
  }
}

}  // namespace spb
