// Host symbolic analysis: see symbolic.hpp for the reference routine each
// function reproduces.  Arrays are 1-based; index 0 of the work vectors below is
// unused so that the reference's subscripts carry over unchanged.
#include "symbolic.hpp"

#include <algorithm>
#include <cstdio>
#include <limits>
#include <stdexcept>

namespace spb {

// ---------------------------------------------------------------------------
// Graph expansion and diagonal handling
// ---------------------------------------------------------------------------

Graph expand_symmetric(int n, const int64_t* colptr, const int32_t* rowind) {
  // ExpandSymmetric (DistSparseMatrixGraph.cpp:929-1084) on one rank:
  //  * every strictly-lower entry (row r, column c) is mirrored into column r;
  //  * mirrored entries are unpacked in source-column order and written
  //    backwards in front of the column's original entries, so a column ends
  //    up as [mirrored rows, descending] [original rows, as given].
  //  The input graph carries sorted = 1 already, so nothing re-sorts it.
  Graph g;
  g.n = n;
  std::vector<int64_t> extra(n + 1, 0);
  for (int c = 1; c <= n; ++c)
    for (int64_t p = colptr[c - 1]; p < colptr[c]; ++p) {
      int r = rowind[p - 1];
      if (r > c) extra[r]++;
    }
  g.colptr.assign(n + 1, 0);
  g.colptr[0] = 1;
  for (int c = 1; c <= n; ++c)
    g.colptr[c] = g.colptr[c - 1] + extra[c] + (colptr[c] - colptr[c - 1]);
  g.rowind.assign(g.colptr[n] - 1, 0);
  // original entries occupy the tail of each new column
  for (int c = 1; c <= n; ++c) {
    int64_t cnt = colptr[c] - colptr[c - 1];
    int64_t dst = g.colptr[c] - 1 - cnt;  // 0-based start of the tail
    for (int64_t k = 0; k < cnt; ++k) g.rowind[dst + k] = rowind[colptr[c - 1] - 1 + k];
  }
  // mirrored entries: the first one lands just before the tail, later ones further left
  std::vector<int64_t> placed(n + 1, 0);
  for (int c = 1; c <= n; ++c)
    for (int64_t p = colptr[c - 1]; p < colptr[c]; ++p) {
      int r = rowind[p - 1];
      if (r > c) {
        int64_t cnt = colptr[r] - colptr[r - 1];
        int64_t pos = g.colptr[r] - 1 - cnt - 1 - placed[r];  // 0-based
        placed[r]++;
        g.rowind[pos] = c;
      }
    }
  return g;
}

void set_keep_diag(Graph& g, bool keep) {
  // SetKeepDiag (DistSparseMatrixGraph.cpp:39-97): removal keeps the order of the
  // remaining entries; insertion puts the diagonal just before the first row
  // greater than the column (or at the end of the column).
  const int n = g.n;
  if (!keep) {
    int64_t pos = 0;
    for (int c = 1; c <= n; ++c) {
      int64_t b = g.colptr[c - 1] - 1, e = g.colptr[c] - 1;
      g.colptr[c - 1] = pos + 1;
      for (int64_t p = b; p < e; ++p)
        if (g.rowind[p] != c) g.rowind[pos++] = g.rowind[p];
    }
    g.rowind.resize(pos);
    g.colptr[n] = pos + 1;
  } else {
    std::vector<int32_t> nr(g.rowind.size() + n);
    int64_t pos = 0;
    for (int c = 1; c <= n; ++c) {
      int64_t b = g.colptr[c - 1] - 1, e = g.colptr[c] - 1;
      g.colptr[c - 1] = pos + 1;
      bool added = false;
      for (int64_t p = b; p < e; ++p) {
        int r = g.rowind[p];
        if (r < c) nr[pos++] = r;
        if (r > c) {
          if (!added) { nr[pos++] = c; added = true; }
          nr[pos++] = r;
        }
      }
      if (!added) nr[pos++] = c;
    }
    nr.resize(pos);
    g.rowind.swap(nr);
    g.colptr[n] = pos + 1;
  }
}

// ---------------------------------------------------------------------------
// Multiple minimum external degree.
//
// A restatement of Liu's quotient-graph MMD as shipped with symPACK
// (genmmd.F:78-185, mmdint.F, mmdelm.F, mmdupd.F, mmdnum.F) with delta = 0 and
// maxint = 2,000,000,000 (ordmmd.F:70-79), in 32-bit integers.  The tie-breaking
// of the result depends on the exact order in which lists and adjacency entries
// are visited, so the control flow follows the reference step by step; the
// label in each comment is the Fortran statement label it corresponds to.
// Index conventions: dforw plays the role of INVP and dbakw of PERM during the
// elimination, exactly as genmmd reuses them.
// ---------------------------------------------------------------------------
namespace {

class MinDegree {
 public:
  MinDegree(int n, const std::vector<int32_t>& xadj1, std::vector<int32_t>& adj1)
      : n_(n), xadj_(xadj1), adj_(adj1),
        dhead_(n + 2, 0), dforw_(n + 2, 0), dbakw_(n + 2, 0), qsize_(n + 2, 0),
        llist_(n + 2, 0), marker_(n + 2, 0) {}

  std::vector<int32_t> run() {
    std::vector<int32_t> invp(n_, 0);
    if (n_ <= 0) return invp;
    init_degree_lists();
    int num = 1;
    // eliminate isolated nodes (genmmd label 100)
    for (int next = dhead_[1]; next > 0;) {
      int node = next;
      next = dforw_[node];
      marker_[node] = kMaxInt;
      dforw_[node] = -num;
      ++num;
    }
    if (num <= n_) {
      tag_ = 1;
      dhead_[1] = 0;
      int mdeg = 2;
      for (;;) {
        // label 300: smallest nonempty degree bucket
        while (dhead_[mdeg] <= 0) ++mdeg;
        const int mdlmt = mdeg + kDelta;
        int ehead = 0;
        bool finished = false;
        // label 500: multiple elimination of independent minimum-degree nodes
        for (;;) {
          int mdnode = dhead_[mdeg];
          if (mdnode <= 0) {
            ++mdeg;
            if (mdeg > mdlmt) break;
            continue;
          }
          // label 600: unlink mdnode from its bucket and number it
          int next = dforw_[mdnode];
          dhead_[mdeg] = next;
          if (next > 0) dbakw_[next] = -mdeg;
          dforw_[mdnode] = -num;
          if (num + qsize_[mdnode] > n_) { finished = true; break; }
          ++tag_;
          if (tag_ >= kMaxInt) reset_tags();
          eliminate(mdnode);
          num += qsize_[mdnode];
          llist_[mdnode] = ehead;
          ehead = mdnode;
        }
        if (finished) break;
        // label 900
        if (num > n_) break;
        update_degrees(ehead, mdeg);
      }
    }
    number_nodes();  // mmdnum
    for (int i = 1; i <= n_; ++i) invp[i - 1] = dforw_[i];
    return invp;
  }

 private:
  static constexpr int kMaxInt = 2000000000;
  static constexpr int kDelta = 0;

  int n_;
  const std::vector<int32_t>& xadj_;  // 1-based (size n+2)
  std::vector<int32_t>& adj_;         // 1-based (size nadj+1); destroyed
  std::vector<int32_t> dhead_, dforw_, dbakw_, qsize_, llist_, marker_;
  int tag_ = 0;

  void reset_tags() {
    tag_ = 1;
    for (int i = 1; i <= n_; ++i)
      if (marker_[i] < kMaxInt) marker_[i] = 0;
  }

  // mmdint: every node starts in the bucket of (its adjacency length + 1);
  // nodes are pushed at the head, so higher-numbered nodes come first.
  void init_degree_lists() {
    for (int node = 1; node <= n_; ++node) {
      dhead_[node] = 0;
      qsize_[node] = 1;
      marker_[node] = 0;
      llist_[node] = 0;
    }
    for (int node = 1; node <= n_; ++node) {
      int ndeg = xadj_[node + 1] - xadj_[node] + 1;
      int fnode = dhead_[ndeg];
      dforw_[node] = fnode;
      dhead_[ndeg] = node;
      if (fnode > 0) dbakw_[fnode] = node;
      dbakw_[node] = -ndeg;
    }
  }

  // mmdelm: turn mdnode into an element and rebuild the quotient graph.
  void eliminate(int mdnode) {
    const int tag = tag_;
    marker_[mdnode] = tag;
    int istrt = xadj_[mdnode], istop = xadj_[mdnode + 1] - 1;
    int elmnt = 0, rloc = istrt, rlmt = istop;
    // label 200: uneliminated neighbours stay in place, eliminated ones are chained
    for (int i = istrt; i <= istop; ++i) {
      int nabor = adj_[i];
      if (nabor == 0) break;
      if (marker_[nabor] >= tag) continue;
      marker_[nabor] = tag;
      if (dforw_[nabor] < 0) {
        llist_[nabor] = elmnt;
        elmnt = nabor;
      } else {
        adj_[rloc++] = nabor;
      }
    }
    // label 300: merge the reach through each adjacent element
    while (elmnt > 0) {
      adj_[rlmt] = -elmnt;
      int link = elmnt;
    scan_element:  // label 400
      {
        int jstrt = xadj_[link], jstop = xadj_[link + 1] - 1;
        for (int j = jstrt; j <= jstop; ++j) {
          int node = adj_[j];
          link = -node;
          if (node < 0) goto scan_element;
          if (node == 0) break;
          if (marker_[node] >= tag || dforw_[node] < 0) continue;
          marker_[node] = tag;
          // label 600: borrow storage of absorbed elements when full
          while (rloc >= rlmt) {
            int l2 = -adj_[rlmt];
            rloc = xadj_[l2];
            rlmt = xadj_[l2 + 1] - 1;
          }
          adj_[rloc++] = node;
        }
      }
      elmnt = llist_[elmnt];  // label 900
    }
    if (rloc <= rlmt) adj_[rloc] = 0;  // label 1000
    // label 1100: for every node of the reachable set
    int link = mdnode;
  scan_reach:
    {
      int rs = xadj_[link], re = xadj_[link + 1] - 1;
      for (int i = rs; i <= re; ++i) {
        int rnode = adj_[i];
        link = -rnode;
        if (rnode < 0) goto scan_reach;
        if (rnode == 0) return;
        // label 1200: remove rnode from the degree structure
        int pvnode = dbakw_[rnode];
        if (pvnode != 0 && pvnode != -kMaxInt) {
          int nxnode = dforw_[rnode];
          if (nxnode > 0) dbakw_[nxnode] = pvnode;
          if (pvnode > 0) dforw_[pvnode] = nxnode;
          if (pvnode < 0) dhead_[-pvnode] = nxnode;
        }
        // label 1300: purge inactive quotient neighbours of rnode
        int jstrt = xadj_[rnode], jstop = xadj_[rnode + 1] - 1;
        int xq = jstrt;
        for (int j = jstrt; j <= jstop; ++j) {
          int nabor = adj_[j];
          if (nabor == 0) break;
          if (marker_[nabor] >= tag) continue;
          adj_[xq++] = nabor;
        }
        int nq = xq - jstrt;
        if (nq <= 0) {
          // label 1500: no active neighbour left -> rnode is indistinguishable from mdnode
          qsize_[mdnode] += qsize_[rnode];
          qsize_[rnode] = 0;
          marker_[rnode] = kMaxInt;
          dforw_[rnode] = -mdnode;
          dbakw_[rnode] = -kMaxInt;
          continue;
        }
        // label 1600: flag for a degree update, add mdnode as an element neighbour
        dforw_[rnode] = nq + 1;
        dbakw_[rnode] = 0;
        adj_[xq++] = mdnode;
        if (xq <= jstop) adj_[xq] = 0;
      }
    }
  }

  // mmdupd: recompute external degrees of nodes touched by the new elements.
  void update_degrees(int ehead, int& mdeg) {
    const int mdeg0 = mdeg + kDelta;
    for (int elmnt = ehead; elmnt > 0; elmnt = llist_[elmnt]) {
      int mtag = tag_ + mdeg0;
      if (mtag >= kMaxInt) {
        reset_tags();
        mtag = tag_ + mdeg0;
      }
      // label 400: split the element's nodes into the two-neighbour list (q2) and the rest (qx)
      int q2head = 0, qxhead = 0, deg0 = 0;
      int link = elmnt;
    scan_elem:
      {
        int is = xadj_[link], ie = xadj_[link + 1] - 1;
        for (int i = is; i <= ie; ++i) {
          int enode = adj_[i];
          link = -enode;
          if (enode < 0) goto scan_elem;
          if (enode == 0) break;
          if (qsize_[enode] == 0) continue;
          deg0 += qsize_[enode];
          marker_[enode] = mtag;
          if (dbakw_[enode] != 0) continue;
          if (dforw_[enode] != 2) {
            llist_[enode] = qxhead;
            qxhead = enode;
          } else {
            llist_[enode] = q2head;
            q2head = enode;
          }
        }
      }
      // label 900: nodes adjacent to exactly two elements/nodes
      for (int enode = q2head; enode > 0; enode = llist_[enode]) {
        if (dbakw_[enode] != 0) continue;
        ++tag_;
        int deg = deg0;
        int istrt = xadj_[enode];
        int nabor = adj_[istrt];
        if (nabor == elmnt) nabor = adj_[istrt + 1];
        int lk = nabor;
        if (dforw_[nabor] >= 0) {
          deg += qsize_[nabor];
        } else {
        scan_second:  // label 1000
          int is = xadj_[lk], ie = xadj_[lk + 1] - 1;
          for (int i = is; i <= ie; ++i) {
            int node = adj_[i];
            lk = -node;
            if (node == enode) continue;
            if (node < 0) goto scan_second;
            if (node == 0) break;
            if (qsize_[node] == 0) continue;
            if (marker_[node] < tag_) {
              marker_[node] = tag_;
              deg += qsize_[node];
              continue;
            }
            // label 1200
            if (dbakw_[node] != 0) continue;
            if (dforw_[node] == 2) {
              // indistinguishable from enode: merge
              qsize_[enode] += qsize_[node];
              qsize_[node] = 0;
              marker_[node] = kMaxInt;
              dforw_[node] = -enode;
              dbakw_[node] = -kMaxInt;
              continue;
            }
            // label 1300: outmatched by enode
            if (dbakw_[node] == 0) dbakw_[node] = -kMaxInt;
          }
        }
        insert_degree(enode, deg, mdeg);  // label 2100
      }
      // label 1600: remaining nodes
      for (int enode = qxhead; enode > 0; enode = llist_[enode]) {
        if (dbakw_[enode] != 0) continue;
        ++tag_;
        int deg = deg0;
        int is = xadj_[enode], ie = xadj_[enode + 1] - 1;
        for (int i = is; i <= ie; ++i) {
          int nabor = adj_[i];
          if (nabor == 0) break;
          if (marker_[nabor] >= tag_) continue;
          marker_[nabor] = tag_;
          if (dforw_[nabor] >= 0) {
            deg += qsize_[nabor];
            continue;
          }
          int lk = nabor;
        scan_el:  // label 1700
          int js = xadj_[lk], je = xadj_[lk + 1] - 1;
          for (int j = js; j <= je; ++j) {
            int node = adj_[j];
            lk = -node;
            if (node < 0) goto scan_el;
            if (node == 0) break;
            if (marker_[node] >= tag_) continue;
            marker_[node] = tag_;
            deg += qsize_[node];
          }
        }
        insert_degree(enode, deg, mdeg);
      }
      tag_ = mtag;  // label 2300
    }
  }

  void insert_degree(int enode, int deg, int& mdeg) {
    deg = deg - qsize_[enode] + 1;
    int fnode = dhead_[deg];
    dforw_[enode] = fnode;
    dbakw_[enode] = -deg;
    if (fnode > 0) dbakw_[fnode] = enode;
    dhead_[deg] = enode;
    if (deg < mdeg) mdeg = deg;
  }

  // mmdnum: number merged nodes right after their representative.
  void number_nodes() {
    std::vector<int32_t>& invp = dforw_;
    std::vector<int32_t>& perm = dbakw_;
    for (int node = 1; node <= n_; ++node)
      perm[node] = (qsize_[node] <= 0) ? invp[node] : -invp[node];
    for (int node = 1; node <= n_; ++node) {
      if (perm[node] > 0) continue;
      int father = node;
      while (perm[father] <= 0) father = -perm[father];
      int root = father;
      int num = perm[root] + 1;
      invp[node] = -num;
      perm[root] = num;
      father = node;
      for (;;) {
        int nextf = -perm[father];
        if (nextf <= 0) break;
        perm[father] = -root;
        father = nextf;
      }
    }
    for (int node = 1; node <= n_; ++node) {
      int num = -invp[node];
      invp[node] = num;
      perm[num] = node;
    }
  }
};

}  // namespace

namespace {

// Breadth-first level structure of the component of root among unmasked nodes
// (ROOTLS, rootls.F).  ls receives the nodes level by level, xls[l] the start of
// level l (0-based positions, xls[nlvl] = component size).  The mask is restored.
int rcm_levels(int root, const Graph& g, std::vector<int8_t>& mask, std::vector<int32_t>& ls,
               std::vector<int32_t>& xls) {
  mask[root] = 0;
  ls[0] = root;
  int nlvl = 0, lvlend = 0, ccsize = 1;
  for (;;) {
    const int lbegin = lvlend;
    lvlend = ccsize;
    xls[nlvl++] = lbegin;
    for (int i = lbegin; i < lvlend; ++i) {
      const int node = ls[i];
      for (int64_t p = g.colptr[node] - 1; p < g.colptr[node + 1] - 1; ++p) {
        const int nbr = g.rowind[p] - 1;
        if (mask[nbr]) {
          ls[ccsize++] = nbr;
          mask[nbr] = 0;
        }
      }
    }
    if (ccsize == lvlend) break;
  }
  xls[nlvl] = lvlend;
  for (int i = 0; i < ccsize; ++i) mask[ls[i]] = 1;
  return nlvl;
}

// Pseudo-peripheral node of root's component (FNROOT, fnroot.F): repeat the level
// structure from the minimum-degree node of the last level (first such node in level
// order) while the number of levels grows.
int rcm_root(int root, const Graph& g, std::vector<int8_t>& mask, std::vector<int32_t>& ls,
             std::vector<int32_t>& xls) {
  int nlvl = rcm_levels(root, g, mask, ls, xls);
  const int ccsize = xls[nlvl];
  if (nlvl == 1 || nlvl == ccsize) return root;
  for (;;) {
    const int jstrt = xls[nlvl - 1];
    int mindeg = ccsize;
    root = ls[jstrt];
    if (ccsize != jstrt + 1) {
      for (int j = jstrt; j < ccsize; ++j) {
        const int node = ls[j];
        int ndeg = 0;
        for (int64_t p = g.colptr[node] - 1; p < g.colptr[node + 1] - 1; ++p) ndeg += mask[g.rowind[p] - 1] > 0;
        if (ndeg < mindeg) {
          root = node;
          mindeg = ndeg;
        }
      }
    }
    const int nunlvl = rcm_levels(root, g, mask, ls, xls);
    if (nunlvl <= nlvl) return root;
    nlvl = nunlvl;
    if (nlvl >= ccsize) return root;
  }
}

}  // namespace

std::vector<int32_t> rcm_order(const Graph& g) {
  const int n = g.n;
  std::vector<int8_t> mask(n, 1);
  std::vector<int32_t> perm(n), xls(n + 1), deg(n), ls(n);
  std::vector<int8_t> seen(n, 0);
  int num = 0;
  for (int i = 0; i < n && num < n; ++i) {
    if (!mask[i]) continue;
    const int root = rcm_root(i, g, mask, ls, xls);
    // degrees within the component among unmasked nodes (DEGREE, degree.F); the
    // breadth-first order it visits leaves perm[num] = root
    int32_t* pm = perm.data() + num;
    pm[0] = root;
    seen[root] = 1;
    int ccsize = 1, lvlend = 0;
    for (;;) {
      const int lbegin = lvlend;
      lvlend = ccsize;
      for (int k = lbegin; k < lvlend; ++k) {
        const int node = pm[k];
        int ideg = 0;
        for (int64_t p = g.colptr[node] - 1; p < g.colptr[node + 1] - 1; ++p) {
          const int nbr = g.rowind[p] - 1;
          if (!mask[nbr]) continue;
          ++ideg;
          if (seen[nbr]) continue;
          seen[nbr] = 1;
          pm[ccsize++] = nbr;
        }
        deg[node] = ideg;
      }
      if (ccsize == lvlend) break;
    }
    for (int k = 0; k < ccsize; ++k) seen[pm[k]] = 0;
    // Cuthill-McKee numbering (RCM, rcm.F): breadth first from the root, the unnumbered
    // neighbours of each node appended in adjacency order and then sorted by increasing
    // degree with a stable insertion sort
    mask[root] = 0;
    if (ccsize > 1) {
      int lnbr = 0;
      lvlend = -1;
      for (;;) {
        const int lbegin = lvlend + 1;
        lvlend = lnbr;
        for (int k = lbegin; k <= lvlend; ++k) {
          const int node = pm[k];
          const int fnbr = lnbr + 1;
          for (int64_t p = g.colptr[node] - 1; p < g.colptr[node + 1] - 1; ++p) {
            const int nbr = g.rowind[p] - 1;
            if (!mask[nbr]) continue;
            mask[nbr] = 0;
            pm[++lnbr] = nbr;
          }
          for (int kk = fnbr + 1; kk <= lnbr; ++kk) {
            const int v = pm[kk];
            int l = kk - 1;
            while (l >= fnbr && deg[pm[l]] > deg[v]) {
              pm[l + 1] = pm[l];
              --l;
            }
            pm[l + 1] = v;
          }
        }
        if (lnbr <= lvlend) break;
      }
      std::reverse(pm, pm + ccsize);  // reverse Cuthill-McKee
    }
    num += ccsize;
  }
  std::vector<int32_t> invp(n);
  for (int k = 0; k < n; ++k) invp[perm[k]] = k + 1;
  return invp;
}

std::vector<int32_t> mmd_order(const Graph& g) {
  const int n = g.n;
  if ((int64_t)g.rowind.size() > (int64_t)std::numeric_limits<int32_t>::max() - 2)
    throw std::runtime_error("graph too large for 32-bit MMD");
  std::vector<int32_t> xadj(n + 2, 0), adj(g.rowind.size() + 1, 0);
  for (int i = 0; i <= n; ++i) xadj[i + 1] = (int32_t)g.colptr[i];
  for (size_t k = 0; k < g.rowind.size(); ++k) adj[k + 1] = g.rowind[k];
  MinDegree md(n, xadj, adj);
  return md.run();
}

// ---------------------------------------------------------------------------
// Elimination tree, postorder, column counts
// ---------------------------------------------------------------------------

std::vector<int32_t> construct_etree(const Graph& g, const std::vector<int32_t>& perm,
                                     const std::vector<int32_t>& invp) {
  // ETree::ConstructETree(SparseMatrixGraph&, ...) ETree.cpp:317-397:
  // Liu's algorithm with path compression on the permuted graph.
  const int n = g.n;
  std::vector<int32_t> parent(n, 0), ancstr(n, 0);
  for (int i = 1; i <= n; ++i) {
    parent[i - 1] = 0;
    ancstr[i - 1] = 0;
    int node = perm[i - 1];
    int64_t jstrt = g.colptr[node - 1], jstop = g.colptr[node] - 1;
    if (jstrt >= jstop) continue;
    for (int64_t j = jstrt; j <= jstop; ++j) {
      int nbr = invp[g.rowind[j - 1] - 1];
      if (nbr >= i) continue;
      if (ancstr[nbr - 1] == i) continue;
      bool stop = false;
      while (ancstr[nbr - 1] > 0) {
        if (ancstr[nbr - 1] == i) { stop = true; break; }
        int next = ancstr[nbr - 1];
        ancstr[nbr - 1] = i;
        nbr = next;
      }
      if (!stop) {
        parent[nbr - 1] = i;
        ancstr[nbr - 1] = i;
      }
    }
  }
  return parent;
}

namespace {
// Depth-first traversal of a first-son / brother tree rooted at n
// (ETree.cpp:24-56 BTreeToPO and its copy inside SortChildren).
std::vector<int32_t> btree_to_postorder(int n, const std::vector<int32_t>& fson,
                                        const std::vector<int32_t>& brother) {
  std::vector<int32_t> stack(n), invpos(n, 0);
  int top = 0, vertex = n, m = 0;
  while (m < n) {
    do {
      stack[top++] = vertex;
      vertex = fson[vertex - 1];
    } while (vertex > 0);
    bool done = false;
    while (vertex == 0) {
      if (top <= 0) { done = true; break; }
      vertex = stack[--top];
      ++m;
      invpos[vertex - 1] = m;
      vertex = brother[vertex - 1];
    }
    if (done) break;
  }
  return invpos;
}

// Ordering::Compose (Ordering.cpp:1301-1315).
void compose(std::vector<int32_t>& perm, std::vector<int32_t>& invp, const std::vector<int32_t>& invp2) {
  const int n = (int)invp.size();
  for (int i = 0; i < n; ++i) invp[i] = invp2[invp[i] - 1];
  for (int i = 1; i <= n; ++i) perm[invp[i - 1] - 1] = i;
}
}  // namespace

std::vector<int32_t> postorder_tree(const std::vector<int32_t>& parent, std::vector<int32_t>& perm,
                                    std::vector<int32_t>& invp) {
  // ETree::PostOrderTree, ETree.cpp:59-119.  Vertex n is taken as the first root;
  // the loop visits n-1 .. 1.
  const int n = (int)parent.size();
  std::vector<int32_t> poparent(n, 0);
  if (n == 0) return poparent;
  std::vector<int32_t> fson(n, 0), brother(n, 0);
  int lroot = n;
  for (int v = n - 1; v > 0; --v) {
    int p = parent[v - 1];
    if (p == 0 || p == v) {
      brother[lroot - 1] = v;
      lroot = v;
    } else {
      brother[v - 1] = fson[p - 1];
      fson[p - 1] = v;
    }
  }
  std::vector<int32_t> invpos = btree_to_postorder(n, fson, brother);
  for (int i = 1; i <= n; ++i) {
    int nu = invpos[i - 1];
    int par = parent[i - 1];
    if (par > 0) par = invpos[par - 1];
    poparent[nu - 1] = par;
  }
  compose(perm, invp, invpos);
  return poparent;
}

void column_counts(const Graph& g, const std::vector<int32_t>& perm, const std::vector<int32_t>& invp,
                   const std::vector<int32_t>& poparent, std::vector<int32_t>& cc,
                   std::vector<int32_t>& rc) {
  // getLColRowCount (symPACKMatrixBase_impl.hpp:310-470): Gilbert-Ng-Peyton
  // row/column counts with path halving.  `level` is unsigned in the reference;
  // the row-count differences wrap the same way here.
  const int n = g.n;
  cc.assign(n, 0);
  rc.assign(n, 0);
  std::vector<uint32_t> level(n + 1), fdesc(n + 1), nchild(n + 1), set(n), prvlf(n), prvnbr(n);
  std::vector<int32_t> weight(n + 1, 0);
  uint32_t xsup = 1;
  level[0] = 0;
  for (int k = n; k >= 1; --k) {
    rc[k - 1] = 1;
    cc[k - 1] = 0;
    set[k - 1] = k;
    prvlf[k - 1] = 0;
    prvnbr[k - 1] = 0;
    level[k] = level[poparent[k - 1]] + 1;
    weight[k] = 1;
    fdesc[k] = k;
    nchild[k] = 0;
  }
  nchild[0] = 0;
  fdesc[0] = 0;
  for (int k = 1; k < n; ++k) {
    uint32_t p = poparent[k - 1];
    weight[p] = 0;
    ++nchild[p];
    if (fdesc[k] < fdesc[p]) fdesc[p] = fdesc[k];
  }
  for (uint32_t low = 1; low <= (uint32_t)n; ++low) {
    int lflag = 0;
    uint32_t ifdesc = fdesc[low];
    int old = perm[low - 1];
    for (int64_t j = g.colptr[old - 1]; j <= g.colptr[old] - 1; ++j) {
      uint32_t hi = invp[g.rowind[j - 1] - 1];
      if (hi <= low) continue;
      if (ifdesc > prvnbr[hi - 1]) {
        ++weight[low];
        uint32_t pleaf = prvlf[hi - 1];
        if (pleaf == 0) {
          rc[hi - 1] = (int32_t)((uint32_t)rc[hi - 1] + (level[low] - level[hi]));
        } else {
          uint32_t last1 = pleaf, last2 = set[last1 - 1], lca = set[last2 - 1];
          while (lca != last2) {
            set[last1 - 1] = lca;
            last1 = lca;
            last2 = set[last1 - 1];
            lca = set[last2 - 1];
          }
          rc[hi - 1] = (int32_t)((uint32_t)rc[hi - 1] + (level[low] - level[lca]));
          --weight[lca];
        }
        prvlf[hi - 1] = low;
        lflag = 1;
      }
      prvnbr[hi - 1] = low;
    }
    uint32_t p = poparent[low - 1];
    --weight[p];
    if (lflag == 1 || nchild[low] >= 2) xsup = low;
    set[xsup - 1] = p;
  }
  for (int k = 1; k <= n; ++k) {
    int t = cc[k - 1] + weight[k];
    cc[k - 1] = t;
    int p = poparent[k - 1];
    if (p != 0) cc[p - 1] += t;
  }
}

void sort_children(std::vector<int32_t>& poparent, std::vector<int32_t>& cc, std::vector<int32_t>& perm,
                   std::vector<int32_t>& invp) {
  // ETree::SortChildren, ETree.cpp:122-225.  Children with a column count at
  // least the current last son's go in front; the postorder is then redone and
  // composed into the ordering, and cc is permuted along.
  const int n = (int)poparent.size();
  if (n == 0) return;
  std::vector<int32_t> fson(n, 0), brother(n, 0), lson(n, 0);
  int lroot = n;
  for (int v = n - 1; v > 0; --v) {
    int p = poparent[v - 1];
    if (p == 0 || p == v) {
      brother[lroot - 1] = v;
      lroot = v;
    } else {
      int ls = lson[p - 1];
      if (ls > 0) {
        if (cc[v - 1] >= cc[ls - 1]) {
          brother[v - 1] = fson[p - 1];
          fson[p - 1] = v;
        } else {
          brother[ls - 1] = v;
          lson[p - 1] = v;
        }
      } else {
        fson[p - 1] = v;
        lson[p - 1] = v;
      }
    }
  }
  brother[lroot - 1] = 0;
  std::vector<int32_t> invpos = btree_to_postorder(n, fson, brother);
  std::vector<int32_t> np(n, 0);
  for (int i = 1; i <= n; ++i) {
    int nu = invpos[i - 1];
    int par = poparent[i - 1];
    if (par > 0) par = invpos[par - 1];
    np[nu - 1] = par;
  }
  poparent = np;
  std::vector<int32_t> tmp(n);
  for (int node = 1; node <= n; ++node) tmp[invpos[node - 1] - 1] = cc[node - 1];
  cc = tmp;
  compose(perm, invp, invpos);
}

// ---------------------------------------------------------------------------
// Supernodes
// ---------------------------------------------------------------------------

void find_supernodes(const std::vector<int32_t>& poparent, const std::vector<int32_t>& cc,
                     std::vector<int32_t>& supmember, std::vector<int32_t>& xsuper, int maxSize) {
  // findSupernodes, symPACKMatrixBase_impl.hpp:42-80 (fundamental supernodes).
  const int n = (int)cc.size();
  supmember.assign(n, 0);
  if (n == 0) { xsuper.assign(1, 1); return; }
  int nsuper = 1, supsize = 1;
  supmember[0] = 1;
  for (int i = 2; i <= n; ++i) {
    int prev_parent = poparent[i - 2];
    if (prev_parent == i && cc[i - 2] == cc[i - 1] + 1 && (supsize < maxSize || maxSize == 0)) {
      ++supsize;
      supmember[i - 1] = nsuper;
      continue;
    }
    ++nsuper;
    supsize = 1;
    supmember[i - 1] = nsuper;
  }
  xsuper.assign(nsuper + 1, 0);
  int lstsup = nsuper + 1;
  for (int i = n; i >= 1; --i) {
    int ksup = supmember[i - 1];
    if (ksup != lstsup) xsuper[lstsup - 1] = i + 1;
    lstsup = ksup;
  }
  xsuper[0] = 1;
}

namespace {
// DisjointSet of ETree.hpp:12-99, including its find() that resets a
// grandparent to be its own parent (makeSet) while walking.
struct RefDisjointSet {
  std::vector<int32_t> pp, root;
  explicit RefDisjointSet(int n) : pp(n, 0), root(n, 0) {}
  int make_set(int i) { pp[i - 1] = i; return i; }
  int link(int s, int t) { pp[s - 1] = t; return t; }
  int find(int i) {
    int p = pp[i - 1], gp = pp[p - 1];
    while (gp != p) {
      i = make_set(gp);
      p = pp[i - 1];
      gp = pp[p - 1];
    }
    return p;
  }
  void unite(int s, int t, int r) {
    int ts = find(t);
    int ss = find(s);
    ss = link(ss, ts);
    root[ss - 1] = (r == -1) ? t : r;
  }
};
}  // namespace

void relax_supernodes(const std::vector<int32_t>& poparent, std::vector<int32_t>& cc,
                      std::vector<int32_t>& supmember, std::vector<int32_t>& xsuper,
                      const RelaxParams& prm) {
  // relaxSupernodes, symPACKMatrixBase_impl.hpp:473-609: merge a supernode into
  // its parent when the parent immediately follows it and the explicit-zero
  // fraction of the merged supernode stays under the size-dependent threshold.
  const int nsuper = (int)xsuper.size() - 1;
  RefDisjointSet sets(nsuper);
  std::vector<int32_t> ncols(nsuper), zeros(nsuper), newcc(nsuper);
  for (int k = nsuper; k >= 1; --k) {
    int cs = sets.make_set(k);
    sets.root[cs - 1] = k;
    int fc = xsuper[k - 1], lc = xsuper[k] - 1;
    ncols[k - 1] = lc - fc + 1;
    zeros[k - 1] = 0;
    newcc[k - 1] = cc[fc - 1];
  }
  for (int k = nsuper; k >= 1; --k) {
    int fc = xsuper[k - 1], lc = xsuper[k] - 1;
    int width = ncols[k - 1];
    int pfc = poparent[lc - 1];
    if (pfc == 0) continue;
    int psn = supmember[pfc - 1];
    int pset = sets.find(psn);
    psn = sets.root[pset - 1];
    if (psn != k + 1) continue;
    int pwidth = ncols[psn - 1];
    int pfirst = xsuper[psn - 1];
    int totzeros = zeros[psn - 1];
    int merged = width + pwidth;
    bool merge = false;
    if ((merged <= prm.maxSize || prm.maxSize == 0) && prm.nrelax0 > 0) {
      if (merged <= prm.nrelax0) {
        merge = true;
      } else if (merged <= prm.maxSize || prm.maxSize == 0) {
        double nnzchild = cc[fc - 1];
        double nnzparent = cc[pfirst - 1];
        double xnewzeros = width * (nnzparent + width - nnzchild);
        if (xnewzeros == 0) {
          merge = true;
        } else {
          double xtotzeros = (double)totzeros + xnewzeros;
          double xm = (double)merged;
          double xtotsize = (xm * (xm + 1) / 2) + xm * (nnzparent - pwidth);
          double z = xtotzeros / xtotsize;
          totzeros += (int)xnewzeros;
          double ptr_max = (double)std::numeric_limits<uint64_t>::max();
          if (xtotsize * sizeof(double) < ptr_max) {
            if (merged <= prm.nrelax1 && z < prm.zrelax0) merge = true;
            else if (merged <= prm.nrelax2 && z < prm.zrelax1) merge = true;
            else if (z < prm.zrelax2) merge = true;
          }
        }
      }
    }
    if (merge) {
      ncols[k - 1] += ncols[psn - 1];
      zeros[k - 1] = totzeros;
      newcc[k - 1] = width + newcc[psn - 1];
      sets.unite(k, psn, k);
    }
  }
  std::vector<int32_t> rx(nsuper + 1);
  int nr = 0;
  for (int k = 1; k <= nsuper; ++k) {
    int ks = sets.find(k);
    if (k == sets.root[ks - 1]) {
      rx[nr] = xsuper[k - 1];
      newcc[nr] = newcc[k - 1];
      ++nr;
    }
  }
  rx[nr] = xsuper[nsuper];
  rx.resize(nr + 1);
  for (int k = 1; k <= nr; ++k) {
    int fc = rx[k - 1], lc = rx[k] - 1;
    for (int c = fc; c <= lc; ++c) {
      supmember[c - 1] = k;
      cc[c - 1] = newcc[k - 1] - (c - fc);
    }
  }
  xsuper = rx;
}

void symbolic_structure(const Graph& g, const std::vector<int32_t>& invp,
                        const std::vector<int32_t>& poparent, const std::vector<int32_t>& cc,
                        const std::vector<int32_t>& xsuper, const std::vector<int32_t>& supmember,
                        std::vector<int64_t>& xlindx, std::vector<int32_t>& lindx) {
  // symbolicFactorizationRelaxedDist on one rank (symPACKMatrixBase_impl.hpp:613-935):
  // the row structure of supernode K is merged, as a sorted linked list, from
  // its children's structures and the permuted columns of A it contains.
  const int n = g.n;
  const int nsuper = (int)xsuper.size() - 1;
  // permuted expanded graph: column invp[c] gets rows invp[r]
  std::vector<int64_t> pcol(n + 1, 0);
  for (int c = 1; c <= n; ++c) pcol[invp[c - 1]] = g.colptr[c] - g.colptr[c - 1];
  std::vector<int64_t> pptr(n + 1, 0);
  for (int c = 1; c <= n; ++c) pptr[c] = pptr[c - 1] + pcol[c];
  std::vector<int32_t> prow(pptr[n]);
  for (int c = 1; c <= n; ++c) {
    int64_t dst = pptr[invp[c - 1] - 1];
    for (int64_t p = g.colptr[c - 1]; p < g.colptr[c]; ++p) prow[dst++] = invp[g.rowind[p - 1] - 1];
  }
  int64_t nofsub = 0;
  for (int k = 1; k <= nsuper; ++k) nofsub += cc[xsuper[k - 1] - 1];
  lindx.assign(nofsub, 0);
  xlindx.assign(nsuper + 1, 0);
  {
    int64_t point = 1;
    for (int k = 1; k <= nsuper; ++k) {
      xlindx[k - 1] = point;
      point += cc[xsuper[k - 1] - 1];
    }
    xlindx[nsuper] = point;
  }
  const uint32_t tail = n + 1, head = 0;
  std::vector<int32_t> mrglnk(nsuper, 0);
  std::vector<uint32_t> rchlnk(n + 1);
  std::vector<int32_t> marker(n, 0);
  int64_t nzend = 0;
  for (int ksup = 1; ksup <= nsuper; ++ksup) {
    int fstcol = xsuper[ksup - 1], lstcol = xsuper[ksup] - 1;
    int width = lstcol - fstcol + 1;
    int length = cc[fstcol - 1];
    int64_t knz = 0;
    rchlnk[head] = tail;
    int jsup = mrglnk[ksup - 1];
    if (jsup > 0) {
      int parentJ = ksup;
      do {
        int jwidth = xsuper[jsup] - xsuper[jsup - 1];
        int64_t jnzbeg = xlindx[jsup - 1] + jwidth, jnzend = xlindx[jsup] - 1;
        if (parentJ == ksup) {
          // first child: copy its structure below its own columns
          for (int64_t jp = jnzend; jp >= jnzbeg; --jp) {
            uint32_t newi = lindx[jp - 1];
            ++knz;
            marker[newi - 1] = ksup;
            rchlnk[newi] = rchlnk[head];
            rchlnk[head] = newi;
          }
        } else {
          // later children: merge into the sorted list
          uint32_t nexti = head;
          for (int64_t jp = jnzbeg; jp <= jnzend; ++jp) {
            uint32_t newi = lindx[jp - 1], i;
            do {
              i = nexti;
              nexti = rchlnk[i];
            } while (newi > nexti);
            if (newi < nexti) {
              ++knz;
              rchlnk[i] = newi;
              rchlnk[newi] = nexti;
              marker[newi - 1] = ksup;
              nexti = newi;
            }
          }
        }
        parentJ = jsup;
        jsup = mrglnk[jsup - 1];
      } while (jsup != 0 && knz < length);
    }
    if (knz < length) {
      auto insert = [&](uint32_t newi) {
        uint32_t nexti = head, i;
        do {
          i = nexti;
          nexti = rchlnk[i];
        } while (newi > nexti);
        ++knz;
        rchlnk[i] = newi;
        rchlnk[newi] = nexti;
        marker[newi - 1] = ksup;
      };
      for (int row = fstcol; row <= lstcol; ++row)
        if (row > fstcol && marker[row - 1] != ksup) insert(row);
      for (int col = fstcol; col <= lstcol; ++col)
        for (int64_t p = pptr[col - 1]; p < pptr[col]; ++p) {
          uint32_t newi = prow[p];
          if ((int)newi > fstcol && marker[newi - 1] != ksup) insert(newi);
        }
    }
    if (rchlnk[head] != (uint32_t)fstcol) {
      rchlnk[fstcol] = rchlnk[head];
      rchlnk[head] = fstcol;
      ++knz;
    }
    if (knz != length) {
      char msg[160];
      snprintf(msg, sizeof msg, "symbolic structure: supernode %d has %lld rows, column count says %d",
               ksup, (long long)knz, length);
      throw std::runtime_error(msg);
    }
    int64_t nzbeg = nzend + 1;
    nzend += knz;
    uint32_t i = head;
    for (int64_t kp = nzbeg; kp <= nzend; ++kp) {
      i = rchlnk[i];
      lindx[kp - 1] = i;
    }
    if (length > width) {
      int pcolumn = poparent[lstcol - 1];
      int psup = supmember[pcolumn - 1];
      mrglnk[ksup - 1] = mrglnk[psup - 1];
      mrglnk[psup - 1] = ksup;
    }
  }
  lindx.resize(nzend);
}

Cells build_cells(const Symbolic& s) {
  // Cell construction of symPACKMatrix2D.hpp:3317-3396: supernodes are visited
  // from the last to the first; each supernode's row list is cut where the
  // owning supernode changes (a cell) and where rows stop being contiguous (a block).
  Cells out;
  const int nsuper = s.nsuper();
  for (int I = nsuper; I >= 1; --I) {
    int64_t lfi = s.xlindx[I - 1], lli = s.xlindx[I] - 1;
    int prevK = -1;
    int start = 0, prev = 0, contig = 0;
    CellBlocks* cur = nullptr;
    auto close_block = [&]() {
      out.block_first_row.push_back(start);
      out.block_nrows.push_back(contig);
      cur->nblocks++;
    };
    for (int64_t p = lfi; p <= lli; ++p) {
      int row = s.lindx[p - 1];
      int K = s.supmember[row - 1];
      if (K != prevK && K >= I) {
        if (cur) close_block();
        out.cells.push_back(CellBlocks{I, K, 0, (int32_t)out.block_first_row.size(), 0});
        cur = &out.cells.back();
        contig = 0;
        start = row;
        prev = row;
      }
      prevK = K;
      if (row == prev + 1 || row == start) {
        ++contig;
      } else {
        close_block();
        contig = 1;
        start = row;
      }
      prev = row;
      cur->nrows++;
    }
    if (cur) close_block();
  }
  return out;
}

// ---------------------------------------------------------------------------
// Driver: symPACKMatrix2D::SymbolicFactorization, MMD branch (2D.hpp:2699-3081)
// ---------------------------------------------------------------------------

Symbolic symbolic_factorization(int n, const int64_t* colptr, const int32_t* rowind,
                                OrderingKind ordering, const RelaxParams& relax,
                                const int32_t* user_perm) {
  if (n <= 0) throw std::invalid_argument("matrix size must be positive");
  if (colptr[0] != 1) throw std::invalid_argument("colptr must be 1-based");
  for (int c = 1; c <= n; ++c) {
    if (colptr[c] < colptr[c - 1]) throw std::invalid_argument("colptr must be nondecreasing");
    for (int64_t p = colptr[c - 1]; p < colptr[c]; ++p) {
      int r = rowind[p - 1];
      if (r < c || r > n) throw std::invalid_argument("rowind must hold lower-triangle rows in [col, n]");
      if (p > colptr[c - 1] && r <= rowind[p - 2])
        throw std::invalid_argument("rows of each column must be strictly increasing");
    }
  }
  Symbolic s;
  s.n = n;
  Graph full = expand_symmetric(n, colptr, rowind);  // keepDiag = 1, sorted flag kept
  Graph sg = full;                                   // GatherStructure at one rank
  if (ordering == OrderingKind::MMD || ordering == OrderingKind::RCM || ordering == OrderingKind::AMD) {
    set_keep_diag(sg, false);
    s.invp = ordering == OrderingKind::MMD ? mmd_order(sg)
             : ordering == OrderingKind::RCM ? rcm_order(sg)
                                             : amd_order(sg);
    set_keep_diag(sg, true);
  } else if (ordering == OrderingKind::NATURAL) {
    s.invp.resize(n);
    for (int i = 0; i < n; ++i) s.invp[i] = i + 1;
  } else {
    if (!user_perm) throw std::invalid_argument("USER ordering needs a permutation");
    s.invp.assign(n, 0);
    for (int i = 0; i < n; ++i) {
      int old = user_perm[i];
      if (old < 1 || old > n || s.invp[old - 1] != 0) throw std::invalid_argument("invalid user permutation");
      s.invp[old - 1] = i + 1;
    }
  }
  s.mmd_invp = s.invp;
  s.perm.assign(n, 0);
  for (int i = 1; i <= n; ++i) s.perm[s.invp[i - 1] - 1] = i;

  std::vector<int32_t> parent = construct_etree(sg, s.perm, s.invp);
  s.parent = postorder_tree(parent, s.perm, s.invp);
  std::vector<int32_t> rc;
  column_counts(sg, s.perm, s.invp, s.parent, s.cc, rc);
  if (ordering != OrderingKind::NATURAL) sort_children(s.parent, s.cc, s.perm, s.invp);
  s.cc_fund = s.cc;
  s.flops_stat = 0.0;
  s.nnzL_stat = 0;
  for (int i = 0; i < n; ++i) {
    s.flops_stat += (double)s.cc[i] * (double)s.cc[i];
    s.nnzL_stat += s.cc[i];
  }
  find_supernodes(s.parent, s.cc, s.supmember, s.xsuper, relax.maxSize);
  if (relax.nrelax0 > 0) relax_supernodes(s.parent, s.cc, s.supmember, s.xsuper, relax);
  symbolic_structure(full, s.invp, s.parent, s.cc, s.xsuper, s.supmember, s.xlindx, s.lindx);
  return s;
}

Symbolic merge_symbolic(const std::vector<Symbolic>& parts) {
  Symbolic m;
  int64_t n = 0, nsup = 0, nl = 0;
  for (const Symbolic& p : parts) {
    n += p.n;
    nsup += p.nsuper();
    nl += (int64_t)p.lindx.size();
  }
  if (n > 2000000000LL) throw std::invalid_argument("batch too large for 32-bit indices");
  m.n = (int)n;
  m.perm.reserve(n);
  m.invp.reserve(n);
  m.mmd_invp.reserve(n);
  m.parent.reserve(n);
  m.cc_fund.reserve(n);
  m.cc.reserve(n);
  m.supmember.reserve(n);
  m.xsuper.reserve(nsup + 1);
  m.xlindx.reserve(nsup + 1);
  m.lindx.reserve(nl);
  int32_t off = 0, soff = 0;
  int64_t loff = 0;
  for (const Symbolic& p : parts) {
    for (int i = 0; i < p.n; ++i) {
      m.perm.push_back(p.perm[i] + off);
      m.invp.push_back(p.invp[i] + off);
      m.mmd_invp.push_back(p.mmd_invp[i] + off);
      m.parent.push_back(p.parent[i] ? p.parent[i] + off : 0);
      m.cc_fund.push_back(p.cc_fund[i]);
      m.cc.push_back(p.cc[i]);
      m.supmember.push_back(p.supmember[i] + soff);
    }
    for (int s = 0; s < p.nsuper(); ++s) {
      m.xsuper.push_back(p.xsuper[s] + off);
      m.xlindx.push_back(p.xlindx[s] + loff);
    }
    for (int32_t r : p.lindx) m.lindx.push_back(r + off);
    m.flops_stat += p.flops_stat;
    m.nnzL_stat += p.nnzL_stat;
    off += p.n;
    soff += p.nsuper();
    loff += (int64_t)p.lindx.size();
  }
  m.xsuper.push_back(off + 1);
  m.xlindx.push_back(loff + 1);
  return m;
}

}  // namespace spb
