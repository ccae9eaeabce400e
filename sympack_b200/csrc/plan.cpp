#include "plan.hpp"

#include <algorithm>
#include <stdexcept>

namespace spb {

static int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

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
  auto push_tiles = [&](std::vector<TileItem>& out, int T, int s, int mode, int rbeg, int rend, int cbeg, int cend,
                        int k0, int kn) {
    for (int cj = cbeg; cj < cend; cj += T)
      for (int ri = rbeg; ri < rend; ri += T) {
        if (ri + T <= cj) continue;  // rows and columns are both panel rows: tile above the diagonal
        TileItem t;
        t.s = s;
        t.mode = mode;
        t.a_row0 = ri;
        t.b_row0 = cj;
        t.k0 = k0;
        t.kn = kn;
        t.mrows = std::min(T, rend - ri);
        t.ncols = std::min(T, cend - cj);
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
      split_k(v, pass ? 1 : 4);
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
      int nslots = 0;
      for (int s : sns) {
        if (!P.is_big[s] || c0 >= P.meta[s].w) continue;
        P.panel_items.push_back(PanelItem{s, c0, std::min(prm.nb, P.meta[s].w - c0), -1, nslots++});
      }
      P.max_diag_slots = std::max(P.max_diag_slots, nslots);
      pd.count = (int32_t)P.panel_items.size() - pd.begin;
      if (pd.count) P.steps.push_back(pd);
      Step pt{StepKind::TrsmRows, (int32_t)P.panel_items.size(), 0, c0, 0, Lane::Chain, blk};
      int slot = 0;
      for (int s : sns) {
        if (!P.is_big[s]) continue;
        const SnMeta& m = P.meta[s];
        if (c0 >= m.w) continue;
        int nbk = std::min(prm.nb, m.w - c0);
        for (int r = c0 + nbk; r < m.h; r += 64) P.panel_items.push_back(PanelItem{s, c0, nbk, r, slot});
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
  // relative indices of the external updates: groups of off-diagonal rows by
  // target, positions found by merging the sorted row lists
  P.row_group.assign(P.rows.size(), -1);
  for (int s = 0; s < ns; ++s) {
    const SnMeta& m = P.meta[s];
    const int32_t* rl = P.rows.data() + m.lidx;
    int r = m.w;
    while (r < m.h) {
      const int t = P.supmember0[rl[r]];
      const SnMeta& mt = P.meta[t];
      const int32_t* tl = P.rows.data() + mt.lidx;
      RelGroup g{t, r, (int64_t)P.rel.size()};
      const int gid = (int)P.groups.size();
      P.groups.push_back(g);
      int q = 0;
      for (int i = r; i < m.h; ++i) {
        while (q < mt.h && tl[q] < rl[i]) ++q;
        if (q == mt.h || tl[q] != rl[i]) throw std::runtime_error("plan: update row missing from its target's structure");
        P.rel.push_back(q);
      }
      int e = r;
      while (e < m.h && P.supmember0[rl[e]] == t) P.row_group[m.lidx + e++] = gid;
      r = e;
    }
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
        // pairs (r, c) of the tile with panel row >= panel column
        double pairs = 0.0;
        for (int c = 0; c < t.ncols; ++c) {
          int lo = std::max(0, t.b_row0 + c - t.a_row0);
          if (lo < t.mrows) pairs += t.mrows - lo;
        }
        f += 2.0 * t.kn * pairs;
      }
    }
    P.step_flops[k] = f;
  }
  for (const SnMeta& m : P.meta) P.solve_sweep_bytes += 8.0 * m.h * m.w;

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
  for (int L = 0; L < H; ++L) {
    int maxsb = 0;
    for (int s : P.level_sn[L]) maxsb = std::max(maxsb, nsb_of(s));
    for (int p = 0; p < maxsb; ++p)
      for (int s : P.level_sn[L]) {
        const SnMeta& m = P.meta[s];
        const int nblk = nblk_of(s), noff = (m.h - m.w + 63) / 64;
        if (p >= nsb_of(s)) continue;
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
  return P;
}

std::vector<int64_t> build_assembly_map(const Symbolic& sym, const Plan& P, const int64_t* colptr,
                                        const int32_t* rowind) {
  const int n = sym.n;
  const int64_t nnz = colptr[n] - 1;
  std::vector<int64_t> dst(nnz);
  for (int c = 1; c <= n; ++c)
    for (int64_t p = colptr[c - 1]; p < colptr[c]; ++p) {
      int r = rowind[p - 1];
      int pr = sym.invp[r - 1] - 1, pc = sym.invp[c - 1] - 1;
      if (pr < pc) std::swap(pr, pc);
      int s = P.supmember0[pc];
      const SnMeta& m = P.meta[s];
      const int32_t* rl = P.rows.data() + m.lidx;
      const int32_t* it = std::lower_bound(rl, rl + m.h, pr);
      if (it == rl + m.h || *it != pr) throw std::runtime_error("assembly: entry outside the symbolic structure");
      dst[p - 1] = m.off + (int64_t)(pc - m.fc) * m.ld + (it - rl);
    }
  return dst;
}

}  // namespace spb
