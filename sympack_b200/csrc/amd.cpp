// Approximate minimum degree ordering, from the algorithm of Amestoy, Davis and Duff
// ("An approximate minimum degree ordering algorithm", SIAM J. Matrix Anal. Appl. 17(4),
// 886-905, 1996): a quotient graph of variables and elements, elimination of a variable of
// least approximate external degree, absorption of the elements adjacent to the pivot into
// the new element, approximate degrees from |Le \ Lme|, mass elimination of variables
// adjacent to the new element only, and indistinguishable variables merged into
// supervariables (candidates found by hashing their adjacency).  The variant is the one
// the reference compiles and calls (src/amdbar.F through Ordering::AMD,
// src/Ordering.cpp:411-520): no dense-row detection, no aggressive absorption.
//
// The permutation must be the reference's bit for bit, so every choice that the
// published algorithm leaves open is made the way that code makes it: the degree lists
// are last-in first-out and the pivot is the first variable of the lowest non-empty list;
// the variables of the new element are collected from the pivot's elements in list
// order, then from its own variables; after the degree update a variable's element list
// becomes [new element, e2 .. ek, e1] and its variable list [v2 .. vm, v1]; the hash key is
// the 32-bit wrapped sum of the surviving entries modulo max(1, n - 1), plus one, and each
// hash bucket is last-in first-out; a variable absorbed into a supervariable, or eliminated
// by mass elimination, is numbered just before the element that finally contains it.
// (Those rules are what the golden tests, made from the reference executed here, pin.)
//
// Layout: each variable keeps its adjacent elements and adjacent variables in two
// vectors, each element its member variables; degree and hash buckets are explicit lists.
// Nothing is compacted: a list shrinks in place when it is pruned.
#include <algorithm>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <vector>

#include "symbolic.hpp"

namespace spb {
namespace {

// Buckets of variables by approximate degree; inserting puts a variable first.
class DegreeBuckets {
 public:
  explicit DegreeBuckets(int n) : first_(n + 2, 0), after_(n + 1, 0), before_(n + 1, 0), at_(n + 1, -1) {}
  void insert(int32_t v, int32_t d) {
    const int32_t f = first_[d];
    after_[v] = f;
    before_[v] = 0;
    if (f) before_[f] = v;
    first_[d] = v;
    at_[v] = d;
  }
  void remove(int32_t v) {
    const int32_t a = after_[v], b = before_[v];
    if (a) before_[a] = b;
    if (b) after_[b] = a;
    else first_[at_[v]] = a;
    at_[v] = -1;
  }
  bool holds(int32_t v) const { return at_[v] >= 0; }
  // the first variable of the lowest non-empty bucket at or above *lo, taken out
  int32_t take_min(int32_t* lo, int32_t top) {
    int32_t d = *lo;
    while (d <= top && !first_[d]) ++d;
    if (d > top) throw std::runtime_error("AMD: no variable left to eliminate");
    *lo = d;
    const int32_t v = first_[d];
    remove(v);
    return v;
  }

 private:
  std::vector<int32_t> first_, after_, before_, at_;
};

enum : int8_t { kVariable = 0, kElement = 1, kAbsorbed = 2 };

class AmdOrdering {
 public:
  explicit AmdOrdering(const Graph& g)
      : n_(g.n), kind_(n_ + 1, kVariable), weight_(n_ + 1, 1), degree_(n_ + 1, 0), mark_(n_ + 1, 1),
        rank_(n_ + 1, 0), parent_(n_ + 1, 0), elems_(n_ + 1), vars_(n_ + 1), members_(n_ + 1), buckets_(n_) {
    for (int v = 1; v <= n_; ++v) {
      vars_[v].assign(g.rowind.begin() + (g.colptr[v - 1] - 1), g.rowind.begin() + (g.colptr[v] - 1));
      degree_[v] = (int32_t)vars_[v].size();
    }
    hash_mod_ = std::max(1, n_ - 1);
    stamp_limit_ = std::numeric_limits<int32_t>::max() - n_;
  }

  std::vector<int32_t> order() {
    for (int v = 1; v <= n_; ++v) {
      if (degree_[v] > 0) {
        buckets_.insert(v, degree_[v]);
      } else {  // no neighbours: an element at once, numbered in index order
        kind_[v] = kElement;
        rank_[v] = ++done_;
        mark_[v] = 0;
        vars_[v].clear();
      }
    }
    while (done_ < n_) eliminate(buckets_.take_min(&min_degree_, n_));
    return final_numbers();
  }

 private:
  int32_t n_;
  int32_t done_ = 0;        // variables eliminated so far (pivots, their supervariables, mass-eliminated)
  int32_t min_degree_ = 1;
  int32_t stamp_ = 2;       // mark value of the current pass; marks below it are stale
  int32_t max_degree_ = 0;  // largest new-element degree so far (stamps advance by it)
  int32_t hash_mod_, stamp_limit_;
  std::vector<int8_t> kind_;
  // weight: supervariable size (negated while the variable is in the new element)
  // degree: approximate external degree of a variable, |Le| (weighted) of an element
  // mark: per element, stamp_ + |Le \ Lme| during a degree update (0 once absorbed)
  // rank: elimination number of an element; parent: where an absorbed variable went
  std::vector<int32_t> weight_, degree_, mark_, rank_, parent_;
  std::vector<std::vector<int32_t>> elems_, vars_, members_;
  DegreeBuckets buckets_;
  std::vector<int32_t> bucket_key_;
  std::vector<std::vector<int32_t>> hash_buckets_;

  void refresh_stamp() {
    if (stamp_ < stamp_limit_) return;
    for (int x = 1; x <= n_; ++x)
      if (mark_[x] != 0) mark_[x] = 1;
    stamp_ = 2;
  }

  // Pivot -> element: its variables and those of its adjacent elements (which it absorbs)
  // become the new element's members, in collection order.
  int32_t collect_new_element(int32_t me, std::vector<int32_t>& lme) {
    int32_t wsum = 0;
    auto take = [&](int32_t v) {
      const int32_t wv = weight_[v];
      if (wv <= 0) return;  // already collected, absorbed or eliminated
      wsum += wv;
      weight_[v] = -wv;
      lme.push_back(v);
      buckets_.remove(v);
    };
    for (int32_t e : elems_[me]) {
      for (int32_t v : members_[e]) take(v);
      // the element is absorbed into the new one: it stays an element (its number is kept)
      // but leaves every list (unmarked)
      parent_[e] = me;
      mark_[e] = 0;
      members_[e].clear();
      members_[e].shrink_to_fit();
    }
    for (int32_t v : vars_[me]) take(v);
    elems_[me].clear();
    vars_[me].clear();
    elems_[me].shrink_to_fit();
    vars_[me].shrink_to_fit();
    return wsum;
  }

  void eliminate(const int32_t me) {
    kind_[me] = kElement;
    rank_[me] = done_ + 1;
    int32_t pivot_weight = weight_[me];
    done_ += pivot_weight;
    weight_[me] = -pivot_weight;
    std::vector<int32_t> lme;
    int32_t lme_degree = collect_new_element(me, lme);
    refresh_stamp();

    // |Le \ Lme| for every element e adjacent to the new element's variables
    for (int32_t v : lme) {
      const int32_t wv = -weight_[v];
      for (int32_t e : elems_[v]) {
        int32_t m = mark_[e];
        if (m >= stamp_) m -= wv;
        else if (m != 0) m = degree_[e] + stamp_ - wv;
        mark_[e] = m;
      }
    }

    // approximate degrees, pruned lists, mass elimination, hash buckets
    if (hash_buckets_.empty()) {
      hash_buckets_.resize((size_t)hash_mod_ + 2);
      bucket_key_.assign(n_ + 1, 0);
    }
    for (int32_t v : lme) {
      int32_t d = 0;
      uint32_t hash = 0;  // wraps like a 32-bit integer sum
      std::vector<int32_t>& E = elems_[v];
      size_t ke = 0;
      for (int32_t e : E)
        if (mark_[e] != 0) {  // still an element (absorbed ones are unmarked)
          d += mark_[e] - stamp_;
          E[ke++] = e;
          hash += (uint32_t)e;
        }
      E.resize(ke);
      std::vector<int32_t>& V = vars_[v];
      size_t kv = 0;
      for (int32_t u : V)
        if (weight_[u] > 0) {  // a variable outside the new element
          d += weight_[u];
          V[kv++] = u;
          hash += (uint32_t)u;
        }
      V.resize(kv);
      if (ke == 0 && kv == 0) {  // adjacent to the new element only: eliminated with it
        kind_[v] = kAbsorbed;
        parent_[v] = me;
        const int32_t wv = -weight_[v];
        lme_degree -= wv;
        pivot_weight += wv;
        done_ += wv;
        weight_[v] = 0;
        E.clear();
        V.clear();
        continue;
      }
      degree_[v] = std::min(degree_[v], d);
      // the new element first, the first surviving element and variable rotate to the back
      if (ke > 0) std::rotate(E.begin(), E.begin() + 1, E.end());
      E.insert(E.begin(), me);
      if (kv > 0) std::rotate(V.begin(), V.begin() + 1, V.end());
      int32_t key = (int32_t)hash % hash_mod_ + 1;
      if (key < 1) key += hash_mod_;  // a negative wrapped sum (not reached by graphs of < 2^31 / n entries)
      hash_buckets_[key].push_back(v);  // read back to front: last in, first out
      bucket_key_[v] = key;
    }
    degree_[me] = lme_degree;
    max_degree_ = std::max(max_degree_, lme_degree);
    stamp_ += max_degree_;
    refresh_stamp();

    // supervariables: variables of one bucket with equal lists merge into the first
    std::vector<int32_t> chain;
    for (int32_t v : lme) {
      if (weight_[v] >= 0) continue;  // mass-eliminated or merged already
      std::vector<int32_t>& bucket = hash_buckets_[bucket_key_[v]];
      if (bucket.empty()) continue;  // bucket done
      chain.assign(bucket.rbegin(), bucket.rend());
      bucket.clear();
      for (size_t a = 0; a + 1 < chain.size(); ++a) {
        const int32_t i = chain[a];
        if (i == 0) continue;
        size_t live = a + 1;  // the scan ends at the bucket's last live variable
        while (live < chain.size() && chain[live] == 0) ++live;
        if (live == chain.size()) break;
        auto tail_of = [&](int32_t x, auto&& f) {  // every list entry but the first (the new element)
          for (size_t q = 1; q < elems_[x].size(); ++q) f(elems_[x][q]);
          for (int32_t u : vars_[x]) f(u);
        };
        tail_of(i, [&](int32_t y) { mark_[y] = stamp_; });
        for (size_t b = a + 1; b < chain.size(); ++b) {
          const int32_t j = chain[b];
          if (j == 0 || elems_[j].size() != elems_[i].size() || vars_[j].size() != vars_[i].size()) continue;
          bool same = true;
          tail_of(j, [&](int32_t y) { same = same && mark_[y] == stamp_; });
          if (!same) continue;
          kind_[j] = kAbsorbed;  // j is indistinguishable from i: merged into it
          parent_[j] = i;
          weight_[i] += weight_[j];
          weight_[j] = 0;
          elems_[j].clear();
          vars_[j].clear();
          chain[b] = 0;
        }
        ++stamp_;
      }
    }

    // final degrees; the new element's surviving variables go back into the buckets
    const int32_t left = n_ - done_;
    std::vector<int32_t>& le = members_[me];
    for (int32_t v : lme) {
      const int32_t wv = -weight_[v];
      if (wv <= 0) continue;
      weight_[v] = wv;
      const int32_t d = std::max(1, std::min(degree_[v] + lme_degree - wv, left - wv));
      buckets_.insert(v, d);
      min_degree_ = std::min(min_degree_, d);
      degree_[v] = d;
      le.push_back(v);
    }
    weight_[me] = pivot_weight + lme_degree;
    if (le.empty()) mark_[me] = 0;
  }

  // Elimination numbers: an absorbed variable is numbered just before the element that
  // finally contains it (its chain of parents is walked, every absorbed variable on the
  // way numbered in walk order and pointed at that element), and the element after all
  // of them.  Returns invp (1-based numbers).
  std::vector<int32_t> final_numbers() {
    std::vector<int32_t> number(n_ + 1, 0), next_rank(rank_);
    for (int v = 1; v <= n_; ++v) {
      if (kind_[v] != kAbsorbed || number[v] != 0) continue;
      int32_t e = parent_[v];
      while (kind_[e] != kElement) e = parent_[e];
      int32_t k = next_rank[e];
      for (int32_t j = v; kind_[j] != kElement;) {
        const int32_t up = parent_[j];
        parent_[j] = e;
        if (kind_[j] == kAbsorbed && number[j] == 0) number[j] = k++;
        j = up;
      }
      next_rank[e] = k;
    }
    std::vector<int32_t> invp(n_);
    for (int v = 1; v <= n_; ++v) invp[v - 1] = kind_[v] == kElement ? next_rank[v] : number[v];
    return invp;
  }
};

}  // namespace

std::vector<int32_t> amd_order(const Graph& g) {
  if (g.n == 0) return {};
  if ((int64_t)g.rowind.size() + g.n >= (int64_t)std::numeric_limits<int32_t>::max())
    throw std::runtime_error("graph too large for 32-bit AMD");
  AmdOrdering amd(g);
  return amd.order();
}

}  // namespace spb
