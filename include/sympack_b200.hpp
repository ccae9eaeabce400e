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

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "sympack_b200.h"

namespace sympack_b200 {

class symPACKMatrix2D {
 public:
  symPACKMatrix2D() = default;
  symPACKMatrix2D(const symPACKMatrix2D&) = delete;
  symPACKMatrix2D& operator=(const symPACKMatrix2D&) = delete;
  ~symPACKMatrix2D() {
    if (h_) spb_destroy(h_);
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
  void Solve(const double* RHS, int nrhs, int rhs_size) { check(spb_solve(need(), RHS, nrhs, rhs_size)); }
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
  std::vector<int64_t> colptr_;
  std::vector<int32_t> rowind_;
};

}  // namespace sympack_b200
