// Approximate minimum degree ordering (Amestoy, Davis & Duff, "An approximate minimum
// degree ordering algorithm", SIAM J. Matrix Anal. Appl. 17(4), 1996) in the variant the
// reference compiles (src/amdbar.F: quotient graph with element absorption, approximate
// external degrees, mass elimination, supervariables found by hashing; no dense-row
// detection and no aggressive absorption), called as Ordering::AMD calls it
// (src/Ordering.cpp:411-520): the expanded graph without diagonal, 32-bit indices, a
// workspace of nnz + n entries (IWLEN = nnz + n, PFREE = nnz + 1, so the quotient graph is
// compacted whenever a new element does not fit), and the inverse permutation taken from
// the final numbering.  Every tie-break (degree-list heads, hash-bucket order, the order
// in which element lists are scanned) follows the reference, so the permutation is the
// reference's bit for bit.
//
// All arrays are 1-based (index 0 unused): 0 is the null link and negative values mark
// absorbed elements and eliminated variables, as in the published algorithm.
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <vector>

#include "symbolic.hpp"

namespace spb {
namespace {

class ApproxMinDegree {
 public:
  explicit ApproxMinDegree(const Graph& g) : n_(g.n) {
    const int64_t nnz = (int64_t)g.rowind.size();
    if (nnz + n_ >= (int64_t)std::numeric_limits<int32_t>::max())
      throw std::runtime_error("graph too large for 32-bit AMD");
    iwlen_ = (int32_t)(nnz + n_);
    pfree_ = (int32_t)nnz + 1;
    const size_t N = (size_t)n_ + 1;
    pe_.assign(N, 0);
    len_.assign(N, 0);
    nv_.assign(N, 0);
    next_.assign(N, 0);
    last_.assign(N, 0);
    head_.assign(N, 0);
    elen_.assign(N, 0);
    degree_.assign(N, 0);
    w_.assign(N, 0);
    iw_.assign((size_t)iwlen_ + 1, 0);
    for (int i = 1; i <= n_; ++i) {
      pe_[i] = (int32_t)g.colptr[i - 1];
      len_[i] = (int32_t)(g.colptr[i] - g.colptr[i - 1]);
    }
    for (int64_t k = 0; k < nnz; ++k) iw_[k + 1] = g.rowind[k];
  }

  std::vector<int32_t> run() {
    hmod_ = std::max(1, n_ - 1);
    wbig_ = std::numeric_limits<int32_t>::max() - n_;
    for (int i = 1; i <= n_; ++i) {
      nv_[i] = 1;
      w_[i] = 1;
      degree_[i] = len_[i];
    }
    for (int i = 1; i <= n_; ++i) {
      if (degree_[i] > 0) {
        push_degree_list(i, degree_[i]);
      } else {  // isolated vertex: numbered first, in index order
        elen_[i] = -(++nel_);
        pe_[i] = 0;
        w_[i] = 0;
      }
    }
    while (nel_ < n_) eliminate(select_pivot());
    return number_variables();
  }

 private:
  int32_t n_, iwlen_, pfree_;
  int32_t nel_ = 0, mindeg_ = 1, wflg_ = 2, dmax_ = 0, hmod_ = 1, wbig_ = 0;
  // pe: start of a variable's / element's list in iw (or -parent once absorbed);
  // len: list length; elen: number of elements at the front of a variable's list
  // (negative order once eliminated); nv: supervariable size (negative while in the
  // pivot element); degree: approximate external degree (element: |Le|);
  // next / last / head: degree lists, reused as hash buckets; w: element marks.
  std::vector<int32_t> pe_, len_, nv_, next_, last_, head_, elen_, degree_, w_, iw_;

  void push_degree_list(int32_t i, int32_t deg) {
    const int32_t inext = head_[deg];
    if (inext != 0) last_[inext] = i;
    next_[i] = inext;
    head_[deg] = i;
  }

  void unlink_degree_list(int32_t i) {
    const int32_t ilast = last_[i], inext = next_[i];
    if (inext != 0) last_[inext] = ilast;
    if (ilast != 0)
      next_[ilast] = inext;
    else
      head_[degree_[i]] = inext;
  }

  void reset_marks_if_needed() {
    if (wflg_ < wbig_) return;
    for (int x = 1; x <= n_; ++x)
      if (w_[x] != 0) w_[x] = 1;
    wflg_ = 2;
  }

  int32_t select_pivot() {
    int32_t deg = mindeg_;
    while (deg <= n_ && head_[deg] <= 0) ++deg;
    if (deg > n_) throw std::runtime_error("AMD: degree lists exhausted early");
    const int32_t me = head_[deg];
    mindeg_ = deg;
    const int32_t inext = next_[me];
    if (inext != 0) last_[inext] = 0;
    head_[deg] = inext;
    return me;
  }

  // Move every live list to the front of iw, in the order the lists appear there,
  // followed by the part of the new element built so far (iw[pme1 .. pfree-1]).  The
  // first entry of each list is parked in pe and replaced by -owner, so that a linear
  // pass can find where each list starts.
  void compact(int32_t& pme1) {
    for (int j = 1; j <= n_; ++j) {
      const int32_t pn = pe_[j];
      if (pn > 0) {
        pe_[j] = iw_[pn];
        iw_[pn] = -j;
      }
    }
    int32_t pdst = 1, psrc = 1;
    const int32_t pend = pme1 - 1;
    while (psrc <= pend) {
      const int32_t j = -iw_[psrc++];
      if (j > 0) {
        iw_[pdst] = pe_[j];
        pe_[j] = pdst++;
        const int32_t lenj = len_[j];
        for (int32_t k = 0; k <= lenj - 2; ++k) iw_[pdst + k] = iw_[psrc + k];
        pdst += lenj - 1;
        psrc += lenj - 1;
      }
    }
    const int32_t p1 = pdst;
    for (int32_t ps = pme1; ps <= pfree_ - 1; ++ps) iw_[pdst++] = iw_[ps];
    pme1 = p1;
    pfree_ = pdst;
  }

  void eliminate(const int32_t me) {
    const int32_t elenme = elen_[me];
    elen_[me] = -(nel_ + 1);
    int32_t nvpiv = nv_[me];
    nel_ += nvpiv;
    nv_[me] = -nvpiv;
    int32_t degme = 0, pme1, pme2, newmem;

    // --- the new element Lme: the pivot's variables plus those of its elements ----
    if (elenme == 0) {  // no adjacent elements: build Lme in place of me's list
      pme1 = pe_[me];
      pme2 = pme1 - 1;
      for (int32_t p = pme1; p <= pme1 + len_[me] - 1; ++p) {
        const int32_t i = iw_[p], nvi = nv_[i];
        if (nvi > 0) {
          degme += nvi;
          nv_[i] = -nvi;
          iw_[++pme2] = i;
          unlink_degree_list(i);
        }
      }
      newmem = 0;
    } else {  // Lme appended at pfree; the elements it covers are absorbed
      int32_t p = pe_[me];
      pme1 = pfree_;
      const int32_t slenme = len_[me] - elenme;
      for (int32_t knt1 = 1; knt1 <= elenme + 1; ++knt1) {
        int32_t e, pj, ln;
        if (knt1 > elenme) {  // last: me's own variables
          e = me;
          pj = p;
          ln = slenme;
        } else {
          e = iw_[p++];
          pj = pe_[e];
          ln = len_[e];
        }
        for (int32_t knt2 = 1; knt2 <= ln; ++knt2) {
          const int32_t i = iw_[pj++], nvi = nv_[i];
          if (nvi <= 0) continue;
          if (pfree_ > iwlen_) {
            // out of room: record how far me's and e's lists have been consumed, compact
            pe_[me] = p;
            len_[me] -= knt1;
            if (len_[me] == 0) pe_[me] = 0;
            pe_[e] = pj;
            len_[e] = ln - knt2;
            if (len_[e] == 0) pe_[e] = 0;
            compact(pme1);
            pj = pe_[e];
            p = pe_[me];
          }
          degme += nvi;
          nv_[i] = -nvi;
          iw_[pfree_++] = i;
          unlink_degree_list(i);
        }
        if (e != me) {  // element e absorbed into me
          pe_[e] = -me;
          w_[e] = 0;
        }
      }
      pme2 = pfree_ - 1;
      newmem = pfree_ - pme1;
    }
    degree_[me] = degme;
    pe_[me] = pme1;
    len_[me] = pme2 - pme1 + 1;
    reset_marks_if_needed();

    // --- w[e] - wflg = |Le \ Lme| for every element e adjacent to Lme ------------------
    for (int32_t pme = pme1; pme <= pme2; ++pme) {
      const int32_t i = iw_[pme], eln = elen_[i];
      if (eln <= 0) continue;
      const int32_t nvi = -nv_[i], wnvi = wflg_ - nvi;
      for (int32_t p = pe_[i]; p <= pe_[i] + eln - 1; ++p) {
        const int32_t e = iw_[p];
        int32_t we = w_[e];
        if (we >= wflg_)
          we -= nvi;
        else if (we != 0)
          we = degree_[e] + wnvi;
        w_[e] = we;
      }
    }

    // --- approximate degrees, pruned lists, mass elimination, hash keys ---------------
    for (int32_t pme = pme1; pme <= pme2; ++pme) {
      const int32_t i = iw_[pme];
      const int32_t p1 = pe_[i], p2 = p1 + elen_[i] - 1;
      int32_t pn = p1, deg = 0;
      uint32_t hash = 0;  // 32-bit sum, wrapping as the reference's INTEGER*4 does
      for (int32_t p = p1; p <= p2; ++p) {
        const int32_t e = iw_[p], we = w_[e];
        if (we != 0) {  // element still alive (absorbed ones have w = 0)
          deg += we - wflg_;
          iw_[pn++] = e;
          hash += (uint32_t)e;
        }
      }
      elen_[i] = pn - p1 + 1;  // + 1 for me, placed first below
      const int32_t p3 = pn;
      for (int32_t p = p2 + 1; p <= p1 + len_[i] - 1; ++p) {
        const int32_t j = iw_[p], nvj = nv_[j];
        if (nvj > 0) {  // variable not in Lme
          deg += nvj;
          iw_[pn++] = j;
          hash += (uint32_t)j;
        }
      }
      if (elen_[i] == 1 && p3 == pn) {
        // i is adjacent to me only: eliminated together with me (mass elimination)
        pe_[i] = -me;
        const int32_t nvi = -nv_[i];
        degme -= nvi;
        nvpiv += nvi;
        nel_ += nvi;
        nv_[i] = 0;
        elen_[i] = 0;
      } else {
        degree_[i] = std::min(degree_[i], deg);
        // me goes to the front of i's list: first variable moves to the end, first
        // element to the first variable's place
        iw_[pn] = iw_[p3];
        iw_[p3] = iw_[p1];
        iw_[p1] = me;
        len_[i] = pn - p1 + 1;
        const int32_t key = (int32_t)hash % hmod_ + 1;
        const int32_t j = head_[key];
        if (j <= 0) {  // bucket kept in head (as -first) while the degree list is empty
          next_[i] = -j;
          head_[key] = -i;
        } else {  // degree list in use: bucket kept in last[] of the list's head
          next_[i] = last_[j];
          last_[j] = i;
        }
        last_[i] = key;
      }
    }
    degree_[me] = degme;
    dmax_ = std::max(dmax_, degme);
    wflg_ += dmax_;
    reset_marks_if_needed();

    // --- supervariables: equal lists within a hash bucket merge into the first --------
    for (int32_t pme = pme1; pme <= pme2; ++pme) {
      int32_t i = iw_[pme];
      if (nv_[i] >= 0) continue;
      const int32_t key = last_[i];
      const int32_t j0 = head_[key];
      if (j0 == 0) continue;
      if (j0 < 0) {
        i = -j0;
        head_[key] = 0;
      } else {
        i = last_[j0];
        last_[j0] = 0;
      }
      while (i != 0 && next_[i] != 0) {
        const int32_t ln = len_[i], eln = elen_[i];
        for (int32_t p = pe_[i] + 1; p <= pe_[i] + ln - 1; ++p) w_[iw_[p]] = wflg_;
        int32_t jlast = i, j = next_[i];
        while (j != 0) {
          bool same = len_[j] == ln && elen_[j] == eln;
          for (int32_t p = pe_[j] + 1; same && p <= pe_[j] + ln - 1; ++p) same = w_[iw_[p]] == wflg_;
          if (same) {  // j is indistinguishable from i: absorb it
            pe_[j] = -i;
            nv_[i] += nv_[j];
            nv_[j] = 0;
            elen_[j] = 0;
            j = next_[j];
            next_[jlast] = j;
          } else {
            jlast = j;
            j = next_[j];
          }
        }
        ++wflg_;
        i = next_[i];
      }
    }

    // --- finalise degrees, put the variables of Lme back in the degree lists ----------
    int32_t p = pme1;
    const int32_t nleft = n_ - nel_;
    for (int32_t pme = pme1; pme <= pme2; ++pme) {
      const int32_t i = iw_[pme], nvi = -nv_[i];
      if (nvi <= 0) continue;
      nv_[i] = nvi;
      const int32_t deg = std::max(1, std::min(degree_[i] + degme - nvi, nleft - nvi));
      push_degree_list(i, deg);
      last_[i] = 0;
      mindeg_ = std::min(mindeg_, deg);
      degree_[i] = deg;
      iw_[p++] = i;
    }
    nv_[me] = nvpiv + degme;
    len_[me] = p - pme1;
    if (len_[me] == 0) {
      pe_[me] = 0;
      w_[me] = 0;
    }
    if (newmem != 0) pfree_ = p;
  }

  // Number the variables that were absorbed into supervariables or mass-eliminated
  // right after the principal variable they were merged into (walking the absorption
  // links, with path compression), and return invp.
  std::vector<int32_t> number_variables() {
    for (int i = 1; i <= n_; ++i) {
      if (elen_[i] != 0) continue;
      int32_t j = -pe_[i];
      while (elen_[j] >= 0) j = -pe_[j];
      const int32_t e = j;
      int32_t k = -elen_[e];
      j = i;
      while (elen_[j] >= 0) {
        const int32_t jnext = -pe_[j];
        pe_[j] = -e;
        if (elen_[j] == 0) elen_[j] = k++;
        j = jnext;
      }
      elen_[e] = -k;
    }
    std::vector<int32_t> invp(n_);
    for (int i = 1; i <= n_; ++i) invp[i - 1] = elen_[i] < 0 ? -elen_[i] : elen_[i];
    return invp;
  }
};

}  // namespace

std::vector<int32_t> amd_order(const Graph& g) {
  if (g.n == 0) return {};
  ApproxMinDegree amd(g);
  return amd.run();
}

}  // namespace spb
