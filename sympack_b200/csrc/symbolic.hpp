// Host symbolic analysis for the supernodal Cholesky path.
//
// Every routine here reproduces, bit for bit, the integer result of the
// corresponding symPACK routine on one rank (symPACK v2.0):
//   expand_symmetric      DistSparseMatrixGraph.cpp:929-1084 (ExpandSymmetric)
//   set_keep_diag         DistSparseMatrixGraph.cpp:39-97    (SetKeepDiag)
//   mmd_order             src/ordmmd.F, genmmd.F, mmdint.F, mmdelm.F, mmdupd.F, mmdnum.F
//                         via Ordering.cpp:103-218 (Ordering::MMD)
//   rcm_order             src/genrcm.F, rcm.F, fnroot.F, rootls.F, degree.F
//                         via Ordering.cpp:221-330 (Ordering::RCM)
//   amd_order (amd.cpp)   src/amdbar.F via Ordering.cpp:411-520 (Ordering::AMD)
//   construct_etree       ETree.cpp:317-397
//   postorder_tree        ETree.cpp:24-119 (BTreeToPO, PostOrderTree)
//   column_counts         symPACKMatrixBase_impl.hpp:310-470 (getLColRowCount)
//   sort_children         ETree.cpp:122-225
//   find_supernodes       symPACKMatrixBase_impl.hpp:42-80
//   relax_supernodes      symPACKMatrixBase_impl.hpp:473-609
//   symbolic_structure    symPACKMatrixBase_impl.hpp:613-935 (symbolicFactorizationRelaxedDist)
//   build_cells           symPACKMatrix2D.hpp:3317-3396 (cell / block construction)
// The driving order is symPACKMatrix2D.hpp:2699-3081 (SymbolicFactorization, MMD branch).
//
// All index arrays are 1-based, as in the reference.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace spb {

// Ashcraft-Grimes relaxation parameters (Types.hpp:22-96).  The run_sympack2D
// driver calls SetMaxSize(0) unless -b is given (utils.hpp:342-348), so the
// defaults a driver-equivalent caller sees are these.
struct RelaxParams {
  int nrelax0 = 8;
  int nrelax1 = 32;
  int nrelax2 = 64;
  int maxSize = 0;
  double zrelax0 = 0.8;
  double zrelax1 = 0.1;
  double zrelax2 = 0.05;
};

// Column-compressed graph, 1-based (colptr[0] == 1).
struct Graph {
  int n = 0;
  std::vector<int64_t> colptr;  // n+1 entries, 1-based positions
  std::vector<int32_t> rowind;  // 1-based vertex ids
};

// Ordering selection (Types.hpp OrderingType; only the ones this path supports).
enum class OrderingKind { MMD = 0, NATURAL = 1, USER = 2, RCM = 3, AMD = 4 };

// Full symbolic result of SymbolicFactorization on one rank.
struct Symbolic {
  int n = 0;
  std::vector<int32_t> perm;      // new -> old (1-based), after postorder + SortChildren
  std::vector<int32_t> invp;      // old -> new (1-based)
  std::vector<int32_t> mmd_invp;  // invp straight out of MMD (before postordering)
  std::vector<int32_t> parent;    // postordered elimination tree, parent[i-1] (0 = root)
  std::vector<int32_t> cc_fund;   // column counts after SortChildren (unrelaxed)
  std::vector<int32_t> cc;        // column counts after relaxation
  std::vector<int32_t> xsuper;    // nsuper+1 first columns (1-based)
  std::vector<int32_t> supmember; // supernode id of each column (1-based)
  std::vector<int64_t> xlindx;    // nsuper+1 (1-based positions into lindx)
  std::vector<int32_t> lindx;     // row structure of each supernode (1-based rows)
  double flops_stat = 0.0;        // sum over j of cc_fund[j]^2 (symPACKMatrix2D.hpp:3009-3016)
  int64_t nnzL_stat = 0;          // sum over j of cc_fund[j]
  int nsuper() const { return (int)xsuper.size() - 1; }
};

// One cell (K, I) of the 2D layout: rows of supernode I's structure that fall in
// supernode K, split into blocks of contiguous rows (symPACKMatrix2D.hpp:3317-3396).
struct CellBlocks {
  int32_t I = 0, K = 0;            // source supernode I (columns), target supernode K (rows)
  int32_t nrows = 0;               // total rows of the cell
  int32_t first_block = 0;         // index into block arrays
  int32_t nblocks = 0;
};
struct Cells {
  std::vector<CellBlocks> cells;          // ordered by I descending, then K ascending (reference order)
  std::vector<int32_t> block_first_row;   // 1-based first row of each block
  std::vector<int32_t> block_nrows;
};

// --- graph helpers ---------------------------------------------------------
// Lower-triangle CSC (1-based, diagonal present, rows sorted) -> full symmetric
// graph in the exact entry order symPACK's ExpandSymmetric leaves behind: for
// column c, the rows < c in DESCENDING order, then the original lower entries.
Graph expand_symmetric(int n, const int64_t* colptr, const int32_t* rowind);
// Remove (keep=false) or insert (keep=true) the diagonal, as SetKeepDiag does.
void set_keep_diag(Graph& g, bool keep);

// --- ordering --------------------------------------------------------------
// Multiple minimum external degree (delta = 0, maxint = 2e9) on an expanded
// graph without diagonal.  Returns invp (old -> new, 1-based).
std::vector<int32_t> mmd_order(const Graph& g_nodiag);
// Reverse Cuthill-McKee (George & Liu's SPARSPAK GENRCM: pseudo-peripheral root per
// connected component, breadth-first numbering with neighbours by increasing degree,
// reversed), on the expanded graph without diagonal in its stored entry order.
// Returns invp (old -> new, 1-based).
std::vector<int32_t> rcm_order(const Graph& g_nodiag);
// Approximate minimum degree (Amestoy, Davis & Duff; the AMDBAR variant: no dense-row
// detection, no aggressive absorption) on the expanded graph without diagonal, with a
// workspace of nnz + n entries.  Returns invp (old -> new, 1-based).
std::vector<int32_t> amd_order(const Graph& g_nodiag);

// --- elimination tree & counts --------------------------------------------
std::vector<int32_t> construct_etree(const Graph& g_diag, const std::vector<int32_t>& perm,
                                     const std::vector<int32_t>& invp);
// Postorders parent in place (returns poparent) and composes perm/invp.
std::vector<int32_t> postorder_tree(const std::vector<int32_t>& parent, std::vector<int32_t>& perm,
                                    std::vector<int32_t>& invp);
void column_counts(const Graph& g_diag, const std::vector<int32_t>& perm,
                   const std::vector<int32_t>& invp, const std::vector<int32_t>& poparent,
                   std::vector<int32_t>& cc, std::vector<int32_t>& rc);
void sort_children(std::vector<int32_t>& poparent, std::vector<int32_t>& cc,
                   std::vector<int32_t>& perm, std::vector<int32_t>& invp);

// --- supernodes ------------------------------------------------------------
void find_supernodes(const std::vector<int32_t>& poparent, const std::vector<int32_t>& cc,
                     std::vector<int32_t>& supmember, std::vector<int32_t>& xsuper, int maxSize);
void relax_supernodes(const std::vector<int32_t>& poparent, std::vector<int32_t>& cc,
                      std::vector<int32_t>& supmember, std::vector<int32_t>& xsuper,
                      const RelaxParams& p);
void symbolic_structure(const Graph& g_diag_expanded, const std::vector<int32_t>& invp,
                        const std::vector<int32_t>& poparent, const std::vector<int32_t>& cc,
                        const std::vector<int32_t>& xsuper, const std::vector<int32_t>& supmember,
                        std::vector<int64_t>& xlindx, std::vector<int32_t>& lindx);
Cells build_cells(const Symbolic& s);

// --- driver ----------------------------------------------------------------
// Whole SymbolicFactorization chain on a lower-triangle CSC (1-based, sorted,
// diagonal present).  user_perm (1-based new->old) is used for USER ordering.
Symbolic symbolic_factorization(int n, const int64_t* colptr, const int32_t* rowind,
                                OrderingKind ordering, const RelaxParams& relax,
                                const int32_t* user_perm = nullptr);

// Batching: the symbolic results of independent systems, merged into the
// symbolic result of their block-diagonal matrix (a forest whose trees are the
// systems' elimination trees, each system's ordering kept as it is).
Symbolic merge_symbolic(const std::vector<Symbolic>& parts);

}  // namespace spb
