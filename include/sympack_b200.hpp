/*
 * sympack_b200.hpp — header-only C++ class over the C ABI with the method names and
 * argument meaning of symPACK's symPACKMatrix2D (include/sympack/symPACKMatrix2D.hpp:
 * Init 2649, SymbolicFactorization 2699, DistributeMatrix 6337, Factorize 6579,
 * Solve 6643, GetSolution 6713; accessors symPACKMatrixBase.hpp:96-103), so that code
 * written against that class switches by changing the type.  Errors are exceptions
 * (std::runtime_error with the library's message) where the C ABI returns status codes.
 *
 * The matrix argument of SymbolicFactorization / DistributeMatrix is any type with the
 * public members symPACK's DistSparseMatrix has at one rank: `size`, `Localg_.colptr`
 * (1-based column pointers), `Localg_.rowind` (1-based rows of the lower triangle with
 * the diagonal, sorted per column) and `nzvalLocal`; overloads take the raw arrays.
 */
#pragma once

#include <algorithm>
#include <cstdint>
#include <iomanip>
#include <iostream>
#include <limits>
#include <ostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "sympack_b200.h"

namespace sympack_b200 {

// Supernode relaxation parameters with the reference's field names, constructors and
// setters (include/sympack/Types.hpp:22-96): a positive maxSize caps every nrelax.
// A default-constructed object has no cap (maxSize 0; the reference leaves maxSize
// unset there), which is also what run_sympack2D sets without -b
// (driver/utils.hpp:341-348: SetMaxSize(0)).
struct RelaxationParameters {
  int nrelax0 = 8, nrelax1 = 32, nrelax2 = 64;
  int maxSize = 0;
  double zrelax0 = 0.8, zrelax1 = 0.1, zrelax2 = 0.05;
  RelaxationParameters() = default;
  explicit RelaxationParameters(int pmaxSize) { SetMaxSize(pmaxSize); }
  RelaxationParameters(int p0, int p1, int p2, int pmaxSize) : nrelax0(p0), nrelax1(p1), nrelax2(p2) {
    SetMaxSize(pmaxSize);
  }
  void SetMaxSize(int pmaxSize) {
    maxSize = pmaxSize;
    if (maxSize > 0) {
      nrelax0 = std::min(nrelax0, maxSize);
      nrelax1 = std::min(nrelax1, maxSize);
      nrelax2 = std::min(nrelax2, maxSize);
    }
  }
  void SetNrelax0(int p) { nrelax0 = maxSize > 0 ? std::min(p, maxSize) : p; }
  void SetNrelax1(int p) { nrelax1 = maxSize > 0 ? std::min(p, maxSize) : p; }
  void SetNrelax2(int p) { nrelax2 = maxSize > 0 ? std::min(p, maxSize) : p; }
};

enum class DecompositionType { LL, LDL };

// The symPACKOptions fields this path reads, under the reference's names
// (include/sympack/Types.hpp:106-201): orderingStr ("MMD", "AMD", "RCM", "NATURAL",
// "USER"), relax, decomposition, perm (USER ordering, 1-based), verbose.  The fields
// after them have no counterpart in the reference and select the device, the
// precision form and its refinement target.  The defaults are the reference
// constructor's (Types.hpp:158-188), relax included: supernodes of at most 150 columns
// (RelaxationParameters(150) and SetMaxSize(150), Types.hpp:173-174) until the caller
// sets another cap, as run_sympack2D does with relax.SetMaxSize.
struct symPACKOptions {
  std::string orderingStr = "MMD";
  RelaxationParameters relax = RelaxationParameters(150);
  DecompositionType decomposition = DecompositionType::LL;
  int* perm = nullptr;
  int verbose = 0;
  int device = 0;                       // CUDA device ordinal; < 0 = host-only (symbolic analysis)
  int precision = SPB_PRECISION_FP64;   // or SPB_PRECISION_FP32_IR
  double ir_tolerance = 1e-12;

  spb_options to_c() const {
    spb_options o;
    spb_default_options(&o);
    if (orderingStr == "MMD") o.ordering = SPB_ORDERING_MMD;
    else if (orderingStr == "NATURAL") o.ordering = SPB_ORDERING_NATURAL;
    else if (orderingStr == "RCM") o.ordering = SPB_ORDERING_RCM;
    else if (orderingStr == "AMD") o.ordering = SPB_ORDERING_AMD;
    else if (orderingStr == "USER") o.ordering = SPB_ORDERING_USER;
    else
      throw std::logic_error("This ordering method is not supported by this solver. Valid options are: "
                             "MMD AMD RCM NATURAL USER");
    o.nrelax0 = relax.nrelax0;
    o.nrelax1 = relax.nrelax1;
    o.nrelax2 = relax.nrelax2;
    o.max_snode = relax.maxSize;
    o.zrelax0 = relax.zrelax0;
    o.zrelax1 = relax.zrelax1;
    o.zrelax2 = relax.zrelax2;
    o.user_perm = perm;
    o.decomposition = decomposition == DecompositionType::LDL ? SPB_DECOMPOSITION_LDL : SPB_DECOMPOSITION_LL;
    o.verbose = verbose;
    o.device = device;
    o.precision = precision;
    o.ir_tolerance = ir_tolerance;
    return o;
  }
};

// The factor as a MATLAB expression, the form of symPACKMatrix2D::DumpMatlab
// (2D.hpp:6762-6854): +sparse([rows],[cols],[values],n,n) over the stored entries of the
// lower triangle, supernode by supernode and row by row, in the permuted ordering
// (1-based), values with 17 significant digits.  xsuper / xlindx / lindx: supernodal
// partition and row structure (1-based); panels: per supernode its h x w panel
// column-major with leading dimension h (spb_get_factor's layout).
inline void write_matlab_sparse(std::ostream& os, int n, const std::vector<int32_t>& xsuper,
                                const std::vector<int64_t>& xlindx, const std::vector<int32_t>& lindx,
                                const double* panels) {
  const int nsuper = (int)xsuper.size() - 1;
  const std::ios_base::fmtflags flags = os.flags();
  const std::streamsize prec = os.precision();
  for (int pass = 0; pass < 3; ++pass) {
    os << (pass == 0 ? "+sparse([" : "],[");
    if (pass == 2) os << std::scientific << std::setprecision(std::numeric_limits<double>::max_digits10 - 1);
    const double* p = panels;
    bool first = true;
    for (int s = 0; s < nsuper; ++s) {
      const int fc = xsuper[s], w = xsuper[s + 1] - xsuper[s];
      const int64_t r0 = xlindx[s] - 1, h = xlindx[s + 1] - xlindx[s];
      for (int64_t i = 0; i < h; ++i)
        for (int j = 0; j < w; ++j) {
          const int row = lindx[r0 + i], col = fc + j;
          if (row < col) continue;  // the diagonal block's upper part is not stored
          if (!first) os << ' ';
          first = false;
          if (pass == 0) os << row;
          else if (pass == 1) os << col;
          else os << p[(int64_t)j * h + i];
        }
      p += h * w;
    }
  }
  os << "]," << n << ',' << n << ")\n";
  os.flags(flags);
  os.precision(prec);
}

class symPACKMatrix2D {
 public:
  symPACKMatrix2D() = default;
  symPACKMatrix2D(const symPACKMatrix2D&) = delete;
  symPACKMatrix2D& operator=(const symPACKMatrix2D&) = delete;
  ~symPACKMatrix2D() {
    if (h_) spb_destroy(h_);
  }

  // symPACKMatrix2D::Init(symPACKOptions&) (2D.hpp:2649).
  void Init(symPACKOptions& options) {
    Init(options.to_c());
    options_ = options;
  }
  // Options as spb_options (spb_default_options gives the reference's defaults).
  void Init(const spb_options& o) {
    if (h_) spb_destroy(h_);
    h_ = nullptr;
    if (spb_create(&o, &h_) != SPB_OK) throw std::runtime_error("sympack_b200: invalid options");
  }
  void Init() {
    spb_options o;
    spb_default_options(&o);
    Init(o);
  }

  void SymbolicFactorization(int32_t n, const int64_t* colptr, const int32_t* rowind) {
    n_ = n;
    check(spb_symbolic(need(), n, colptr, rowind));
  }
  template <class DSM>
  void SymbolicFactorization(const DSM& A) {
    colptr_.assign(A.Localg_.colptr.begin(), A.Localg_.colptr.end());
    rowind_.assign(A.Localg_.rowind.begin(), A.Localg_.rowind.end());
    SymbolicFactorization((int32_t)A.size, colptr_.data(), rowind_.data());
  }

  void DistributeMatrix(const double* nzval) { check(spb_distribute(need(), nzval)); }
  template <class DSM>
  void DistributeMatrix(const DSM& A) {
    DistributeMatrix(A.nzvalLocal.data());
  }

  void Factorize() { check(spb_factorize(need())); }

  // RHS column-major n x nrhs with leading dimension rhs_size (>= n), original ordering.
  // Xptr is accepted for the signature of symPACKMatrixMeta::Solve (symPACKMatrixBase.hpp:62);
  // the reference's 2D solver does not use it (2D.hpp:6643-6711) and neither does this one:
  // the solution stays in the object until GetSolution.
  void Solve(const double* RHS, int nrhs, int rhs_size, double* Xptr = nullptr) {
    (void)Xptr;
    check(spb_solve(need(), RHS, nrhs, rhs_size));
  }
  void Solve(const double* RHS, int nrhs) { Solve(RHS, nrhs, n_); }
  void GetSolution(double* B, int nrhs, int ldb) { check(spb_get_solution(need(), B, nrhs, ldb)); }
  void GetSolution(double* B, int nrhs) { GetSolution(B, nrhs, n_); }

  // Accessors (1-based, as the reference's).
  std::vector<int32_t> GetOrdering(std::vector<int32_t>* invp = nullptr) {
    std::vector<int32_t> perm(n_), iv(n_);
    check(spb_get_ordering(need(), perm.data(), iv.data()));
    if (invp) *invp = iv;
    return perm;
  }
  std::vector<int32_t> GetETree() {
    std::vector<int32_t> parent(n_);
    check(spb_get_etree(need(), parent.data()));
    return parent;
  }
  std::vector<int32_t> GetSupernodalPartition() {
    std::vector<int32_t> xsuper(info().nsuper + 1), sup(n_);
    check(spb_get_supernodes(need(), xsuper.data(), sup.data()));
    return xsuper;
  }
  std::vector<int32_t> GetSupMembership() {
    std::vector<int32_t> xsuper(info().nsuper + 1), sup(n_);
    check(spb_get_supernodes(need(), xsuper.data(), sup.data()));
    return sup;
  }
  // symPACKMatrixMeta accessors (symPACKMatrixBase.hpp:96-103): order of the matrix, the
  // options given to Init, number of supernodes.
  int Size() const { return n_; }
  symPACKOptions GetOptions() const { return options_; }
  int TotalSupernodeCnt() { return n_ ? info().nsuper : 0; }

  // symPACKMatrix2D::DumpMatlab (2D.hpp:6762-6854), after Factorize: the factor as
  // +sparse([rows],[cols],[values],n,n) (write_matlab_sparse) on os.
  void DumpMatlab(std::ostream& os = std::cout) {
    const spb_info inf = info();
    std::vector<int32_t> xsuper(inf.nsuper + 1), lindx(inf.lindx_size);
    std::vector<int64_t> xlindx(inf.nsuper + 1);
    check(spb_get_supernodes(need(), xsuper.data(), nullptr));
    check(spb_get_structure(need(), xlindx.data(), lindx.data()));
    size_t total = 0;
    for (int s = 0; s < inf.nsuper; ++s)
      total += (size_t)(xlindx[s + 1] - xlindx[s]) * (size_t)(xsuper[s + 1] - xsuper[s]);
    std::vector<double> panels(total);
    check(spb_get_factor(need(), panels.data()));
    write_matlab_sparse(os, n_, xsuper, xlindx, lindx, panels.data());
  }

  spb_info info() {
    spb_info i;
    check(spb_get_info(need(), &i));
    return i;
  }
  spb_handle* handle() { return h_; }

 private:
  spb_handle* need() {
    if (!h_) throw std::runtime_error("sympack_b200: call Init first");
    return h_;
  }
  void check(int rc) {
    if (rc != SPB_OK) throw std::runtime_error(std::string("sympack_b200: ") + spb_last_error(h_));
  }
  spb_handle* h_ = nullptr;
  int32_t n_ = 0;
  symPACKOptions options_;
  std::vector<int64_t> colptr_;
  std::vector<int32_t> rowind_;
};

}  // namespace sympack_b200
