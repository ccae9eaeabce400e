// Rutherford-Boeing (Harwell-Boeing) input boundary.
//
// spb_rb_read restates ReadHB_PARA on one rank (include/sympack/utility.hpp:1274-1481):
// four header lines (title; card counts; type and dimensions; the Fortran
// formats "(nIw)" "(nIw)" "(nEw.d)"), then colptr, rowind and values read as
// whitespace-separated fields, and finally each column's rows sorted together
// with their values (utility.hpp:1463-1475).  spb_rb_write produces files in the
// fixed-width layout that reader's byte-offset arithmetic assumes: every full
// line holds exactly the format's count of fields of exactly its width.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/sympack_b200.h"

namespace {

struct RbData {
  int32_t n = 0;
  int64_t nnz = 0;
  std::vector<int64_t> colptr;
  std::vector<int32_t> rowind;
  std::vector<double> val;
};

int read_rb(const char* path, RbData& d, bool values) {
  std::ifstream in(path);
  if (!in) return SPB_ERR_INVALID;
  std::string line;
  if (!std::getline(in, line)) return SPB_ERR_INVALID;  // title
  if (!std::getline(in, line)) return SPB_ERR_INVALID;  // card counts
  if (!std::getline(in, line)) return SPB_ERR_INVALID;  // type, nrow, ncol, nnz
  {
    std::istringstream iss(line);
    std::string type;
    long long m = 0, n = 0, nnz = 0;
    iss >> type >> m >> n >> nnz;
    if (!iss || m != n || n <= 0 || nnz < n || n > 2147483647LL) return SPB_ERR_INVALID;
    d.n = (int32_t)n;
    d.nnz = nnz;
  }
  if (!std::getline(in, line)) return SPB_ERR_INVALID;  // formats
  d.colptr.resize(d.n + 1);
  d.rowind.resize(d.nnz);
  for (int64_t i = 0; i <= d.n; ++i)
    if (!(in >> d.colptr[i])) return SPB_ERR_INVALID;
  for (int64_t i = 0; i < d.nnz; ++i) {
    long long r;
    if (!(in >> r)) return SPB_ERR_INVALID;
    d.rowind[i] = (int32_t)r;
  }
  if (d.colptr[0] != 1 || d.colptr[d.n] != d.nnz + 1) return SPB_ERR_INVALID;
  if (values) {
    d.val.resize(d.nnz);
    std::string tok;
    for (int64_t i = 0; i < d.nnz; ++i) {
      if (!(in >> tok)) return SPB_ERR_INVALID;
      for (char& ch : tok)
        if (ch == 'D' || ch == 'd') ch = 'E';
      char* end = nullptr;
      d.val[i] = std::strtod(tok.c_str(), &end);
      if (end == tok.c_str()) return SPB_ERR_INVALID;
    }
  }
  // sort each column's rows (and values) ascending
  std::vector<size_t> idx;
  std::vector<int32_t> rtmp;
  std::vector<double> vtmp;
  for (int32_t c = 0; c < d.n; ++c) {
    int64_t b = d.colptr[c] - 1, e = d.colptr[c + 1] - 1;
    if (e < b) return SPB_ERR_INVALID;
    if (std::is_sorted(d.rowind.begin() + b, d.rowind.begin() + e)) continue;
    idx.resize(e - b);
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return d.rowind[b + x] < d.rowind[b + y]; });
    rtmp.resize(e - b);
    for (size_t k = 0; k < idx.size(); ++k) rtmp[k] = d.rowind[b + idx[k]];
    std::copy(rtmp.begin(), rtmp.end(), d.rowind.begin() + b);
    if (values) {
      vtmp.resize(e - b);
      for (size_t k = 0; k < idx.size(); ++k) vtmp[k] = d.val[b + idx[k]];
      std::copy(vtmp.begin(), vtmp.end(), d.val.begin() + b);
    }
  }
  return SPB_OK;
}

}  // namespace

extern "C" {

int spb_rb_info(const char* path, int32_t* n, int64_t* nnz) {
  if (!path || !n || !nnz) return SPB_ERR_INVALID;
  RbData d;
  int rc = read_rb(path, d, false);
  if (rc) return rc;
  *n = d.n;
  *nnz = d.nnz;
  return SPB_OK;
}

int spb_rb_read(const char* path, int64_t* colptr, int32_t* rowind, double* nzval) {
  if (!path || !colptr || !rowind) return SPB_ERR_INVALID;
  RbData d;
  int rc = read_rb(path, d, nzval != nullptr);
  if (rc) return rc;
  std::copy(d.colptr.begin(), d.colptr.end(), colptr);
  std::copy(d.rowind.begin(), d.rowind.end(), rowind);
  if (nzval) std::copy(d.val.begin(), d.val.end(), nzval);
  return SPB_OK;
}

int spb_rb_write(const char* path, const char* title, int32_t n, const int64_t* colptr, const int32_t* rowind,
                 const double* nzval) {
  if (!path || n <= 0 || !colptr || !rowind || !nzval) return SPB_ERR_INVALID;
  const int64_t nnz = colptr[n] - 1;
  if (nnz + 1 >= 1000000000LL) return SPB_ERR_INVALID;  // I10 fields must keep a separating blank
  FILE* f = std::fopen(path, "w");
  if (!f) return SPB_ERR_INVALID;
  const int ipl = 8, vpl = 4;  // (8I10) and (4E20.12)
  const int64_t ptrcrd = (n + 1 + ipl - 1) / ipl, indcrd = (nnz + ipl - 1) / ipl, valcrd = (nnz + vpl - 1) / vpl;
  char t[73];
  std::snprintf(t, sizeof t, "%-72.72s", title ? title : "");
  std::fprintf(f, "%s%-8.8s\n", t, "spb_rb");
  std::fprintf(f, "%14lld%14lld%14lld%14lld%14d\n", (long long)(ptrcrd + indcrd + valcrd), (long long)ptrcrd,
               (long long)indcrd, (long long)valcrd, 0);
  std::fprintf(f, "%-14s%14d%14d%14lld%14d\n", "rsa", n, n, (long long)nnz, 0);
  std::fprintf(f, "%-16s%-16s%-20s\n", "(8I10)", "(8I10)", "(4E20.12)");
  auto ints = [&](auto get, int64_t count) {
    for (int64_t i = 0; i < count; ++i) {
      std::fprintf(f, "%10lld", (long long)get(i));
      if ((i + 1) % ipl == 0 || i + 1 == count) std::fputc('\n', f);
    }
  };
  ints([&](int64_t i) { return colptr[i]; }, n + 1);
  ints([&](int64_t i) { return (int64_t)rowind[i]; }, nnz);
  for (int64_t i = 0; i < nnz; ++i) {
    std::fprintf(f, "%20.12E", nzval[i]);
    if ((i + 1) % vpl == 0 || i + 1 == nnz) std::fputc('\n', f);
  }
  return std::fclose(f) == 0 ? SPB_OK : SPB_ERR_INVALID;
}

}  // extern "C"
