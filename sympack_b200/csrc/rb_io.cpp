// Rutherford-Boeing (Harwell-Boeing) input boundary.
//
// spb_rb_read restates ReadHB_PARA (include/sympack/utility.hpp:1274-1481): four header
// lines (title; card counts; type and dimensions; the Fortran formats "(nIw)" "(nIw)"
// "(nEw.d)"), then colptr, rowind and values, and finally each column's rows sorted
// together with their values (utility.hpp:1463-1475).  Like the reference, which gives
// each MPI rank a range of columns and finds its bytes by the fixed-width arithmetic
// "field i of a section sits at i * width + i / fields_per_line" (utility.hpp:1352-1360),
// the reader splits every section among host threads by that arithmetic and parses the
// fields in place; it checks first that every line of the file ends where the layout
// says, and reads any other layout (uneven lines, other whitespace) with a sequential
// whitespace-separated parser instead.  spb_rb_write produces the fixed-width layout,
// formatting the sections in parallel into one buffer.
#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <sstream>
#include <string>
#include <thread>
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

struct Section {
  int64_t count = 0;  // fields
  int per = 0;        // fields per full line
  int width = 0;      // characters per field
  size_t start = 0;   // byte offset of the first field
  size_t bytes() const { return (size_t)count * width + (size_t)((count + per - 1) / per); }  // with newlines
  size_t at(int64_t i) const { return start + (size_t)i * width + (size_t)(i / per); }
};

struct Header {
  int32_t n = 0;
  int64_t nnz = 0;
  Section ptr, ind, val;
  size_t data = 0;  // byte offset after the header lines
};

int nthreads_for(int64_t work) {
  const int hw = std::max(1u, std::thread::hardware_concurrency());
  return (int)std::max<int64_t>(1, std::min<int64_t>(std::min(hw, 64), work / 200000));
}

template <class F>
void parallel_ranges(int64_t count, int nt, F f) {
  if (nt <= 1) {
    f(0, count);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) {
    const int64_t b = count * t / nt, e = count * (t + 1) / nt;
    th.emplace_back([=]() { f(b, e); });
  }
  for (auto& x : th) x.join();
}

bool next_line(const std::string& buf, size_t& pos, std::string& line) {
  if (pos >= buf.size()) return false;
  size_t e = buf.find('\n', pos);
  if (e == std::string::npos) e = buf.size();
  line.assign(buf, pos, e - pos);
  if (!line.empty() && line.back() == '\r') line.pop_back();
  pos = e + 1;
  return true;
}

int read_file(const char* path, std::string& buf) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return SPB_ERR_INVALID;
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz < 0) {
    std::fclose(f);
    return SPB_ERR_INVALID;
  }
  buf.resize((size_t)sz);
  const size_t got = sz ? std::fread(&buf[0], 1, (size_t)sz, f) : 0;
  std::fclose(f);
  return got == (size_t)sz ? SPB_OK : SPB_ERR_INVALID;
}

// Header lines; the formats line gives each section's fields per line and width.
int parse_header(const std::string& buf, Header& h) {
  size_t pos = 0;
  std::string line;
  if (!next_line(buf, pos, line)) return SPB_ERR_INVALID;  // title
  if (!next_line(buf, pos, line)) return SPB_ERR_INVALID;  // card counts
  long long totcrd = 0, ptrcrd = 0, indcrd = 0, valcrd = 0, rhscrd = 0;
  {
    std::istringstream iss(line);
    iss >> totcrd >> ptrcrd >> indcrd >> valcrd;
    if (!(iss >> rhscrd)) rhscrd = 0;
  }
  if (!next_line(buf, pos, line)) return SPB_ERR_INVALID;  // type, nrow, ncol, nnz
  {
    std::istringstream iss(line);
    std::string type;
    long long m = 0, n = 0, nnz = 0;
    iss >> type >> m >> n >> nnz;
    if (!iss || m != n || n <= 0 || nnz < n || n > 2147483647LL) return SPB_ERR_INVALID;
    h.n = (int32_t)n;
    h.nnz = nnz;
  }
  if (!next_line(buf, pos, line)) return SPB_ERR_INVALID;  // formats
  {
    std::istringstream iss(line);
    std::string f1, f2, f3;
    iss >> f1 >> f2 >> f3;
    int d = 0;
    if (std::sscanf(f1.c_str(), "(%dI%d)", &h.ptr.per, &h.ptr.width) != 2) h.ptr.per = 0;
    if (std::sscanf(f2.c_str(), "(%dI%d)", &h.ind.per, &h.ind.width) != 2) h.ind.per = 0;
    if (std::sscanf(f3.c_str(), "(%dE%d.%d)", &h.val.per, &h.val.width, &d) != 3 &&
        std::sscanf(f3.c_str(), "(%dD%d.%d)", &h.val.per, &h.val.width, &d) != 3)
      h.val.per = 0;
  }
  if (rhscrd > 0 && !next_line(buf, pos, line)) return SPB_ERR_INVALID;  // right-hand side format line
  h.data = pos;
  h.ptr.count = (int64_t)h.n + 1;
  h.ind.count = h.nnz;
  h.val.count = h.nnz;
  return SPB_OK;
}

// Every line of every section ends exactly where the fixed-width layout puts it.
bool fixed_layout(const std::string& buf, Header& h, bool values) {
  Section* secs[3] = {&h.ptr, &h.ind, &h.val};
  size_t pos = h.data;
  for (int k = 0; k < (values ? 3 : 2); ++k) {
    Section& s = *secs[k];
    if (s.per <= 0 || s.width <= 0 || s.width > 40) return false;
    s.start = pos;
    const int64_t lines = (s.count + s.per - 1) / s.per;
    if (pos + s.bytes() > buf.size()) return false;
    for (int64_t l = 0; l < lines; ++l) {
      const int64_t last = std::min(s.count, (l + 1) * s.per) - 1;  // last field of the line
      if (buf[s.at(last) + s.width] != '\n') return false;
    }
    pos += s.bytes();
  }
  return true;
}

bool parse_int(const char* p, int w, long long& out) {
  int i = 0;
  while (i < w && p[i] == ' ') ++i;
  bool neg = false;
  if (i < w && (p[i] == '-' || p[i] == '+')) neg = p[i++] == '-';
  if (i == w) return false;
  long long v = 0;
  for (; i < w; ++i) {
    if (p[i] < '0' || p[i] > '9') return false;
    v = v * 10 + (p[i] - '0');
  }
  out = neg ? -v : v;
  return true;
}

bool parse_real(const char* p, int w, double& out) {
  char tmp[48];
  int i = 0, k = 0;
  while (i < w && p[i] == ' ') ++i;
  if (i < w && p[i] == '+') ++i;  // from_chars takes no leading '+'
  for (; i < w; ++i) tmp[k++] = (p[i] == 'D' || p[i] == 'd') ? 'E' : p[i];
  while (k > 0 && tmp[k - 1] == ' ') --k;
  if (k == 0) return false;
  const auto r = std::from_chars(tmp, tmp + k, out);
  return r.ec == std::errc() && r.ptr == tmp + k;
}

int read_fixed(const std::string& buf, const Header& h, RbData& d, bool values) {
  const int nt = nthreads_for(h.nnz);
  std::vector<char> bad(nt, 0);
  auto run = [&](const Section& s, auto store) {
    const int ntt = s.count >= 200000 ? nt : 1;
    std::vector<std::thread> th;
    for (int t = 0; t < ntt; ++t) {
      const int64_t b = s.count * t / ntt, e = s.count * (t + 1) / ntt;
      auto body = [&, t, b, e]() {
        for (int64_t i = b; i < e; ++i)
          if (!store(i, buf.data() + s.at(i), s.width)) {
            bad[t] = 1;
            return;
          }
      };
      if (ntt == 1) body();
      else th.emplace_back(body);
    }
    for (auto& x : th) x.join();
  };
  run(h.ptr, [&](int64_t i, const char* p, int w) {
    long long v;
    if (!parse_int(p, w, v)) return false;
    d.colptr[i] = v;
    return true;
  });
  run(h.ind, [&](int64_t i, const char* p, int w) {
    long long v;
    if (!parse_int(p, w, v) || v < 1 || v > d.n) return false;
    d.rowind[i] = (int32_t)v;
    return true;
  });
  if (values) run(h.val, [&](int64_t i, const char* p, int w) { return parse_real(p, w, d.val[i]); });
  for (char b : bad)
    if (b) return SPB_ERR_INVALID;
  return SPB_OK;
}

// Sequential whitespace-separated fields, for layouts that are not fixed-width.
int read_free(const std::string& buf, const Header& h, RbData& d, bool values) {
  std::istringstream in(buf.substr(h.data));
  for (int64_t i = 0; i <= d.n; ++i)
    if (!(in >> d.colptr[i])) return SPB_ERR_INVALID;
  for (int64_t i = 0; i < d.nnz; ++i) {
    long long r;
    if (!(in >> r) || r < 1 || r > d.n) return SPB_ERR_INVALID;
    d.rowind[i] = (int32_t)r;
  }
  if (values) {
    std::string tok;
    for (int64_t i = 0; i < d.nnz; ++i) {
      if (!(in >> tok)) return SPB_ERR_INVALID;
      if (!parse_real(tok.c_str(), (int)tok.size(), d.val[i])) return SPB_ERR_INVALID;
    }
  }
  return SPB_OK;
}

int read_rb(const char* path, RbData& d, bool values) {
  std::string buf;
  int rc = read_file(path, buf);
  if (rc) return rc;
  Header h;
  rc = parse_header(buf, h);
  if (rc) return rc;
  d.n = h.n;
  d.nnz = h.nnz;
  d.colptr.resize(d.n + 1);
  d.rowind.resize(d.nnz);
  if (values) d.val.resize(d.nnz);
  rc = fixed_layout(buf, h, values) ? read_fixed(buf, h, d, values) : read_free(buf, h, d, values);
  if (rc) return rc;
  if (d.colptr[0] != 1 || d.colptr[d.n] != d.nnz + 1) return SPB_ERR_INVALID;
  for (int32_t c = 0; c < d.n; ++c)
    if (d.colptr[c + 1] < d.colptr[c]) return SPB_ERR_INVALID;
  // sort each column's rows (and values) ascending, columns split among threads
  std::vector<char> bad(1, 0);
  parallel_ranges(d.n, nthreads_for(d.nnz), [&](int64_t c0, int64_t c1) {
    std::vector<size_t> idx;
    std::vector<int32_t> rtmp;
    std::vector<double> vtmp;
    for (int64_t c = c0; c < c1; ++c) {
      const int64_t b = d.colptr[c] - 1, e = d.colptr[c + 1] - 1;
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
  });
  return SPB_OK;
}

void put_int(char* p, int w, long long v) {  // right-aligned in w characters
  char tmp[24];
  int k = 0;
  const bool neg = v < 0;
  unsigned long long u = neg ? 0ULL - (unsigned long long)v : (unsigned long long)v;
  do {
    tmp[k++] = (char)('0' + u % 10);
    u /= 10;
  } while (u);
  if (neg) tmp[k++] = '-';
  std::memset(p, ' ', w - k);
  for (int i = 0; i < k; ++i) p[w - 1 - i] = tmp[i];
}

}  // namespace

extern "C" {

int spb_rb_info(const char* path, int32_t* n, int64_t* nnz) {
  if (!path || !n || !nnz) return SPB_ERR_INVALID;
  std::string buf;
  int rc = read_file(path, buf);
  if (rc) return rc;
  Header h;
  rc = parse_header(buf, h);
  if (rc) return rc;
  *n = h.n;
  *nnz = h.nnz;
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
  const int ipl = 8, vpl = 4, iw = 10, vw = 20;  // (8I10) and (4E20.12)
  const int64_t ptrcrd = (n + 1 + ipl - 1) / ipl, indcrd = (nnz + ipl - 1) / ipl, valcrd = (nnz + vpl - 1) / vpl;
  std::string head;
  {
    char t[73], line[128];
    std::snprintf(t, sizeof t, "%-72.72s", title ? title : "");
    head += t;
    std::snprintf(line, sizeof line, "%-8.8s\n", "spb_rb");
    head += line;
    std::snprintf(line, sizeof line, "%14lld%14lld%14lld%14lld%14d\n", (long long)(ptrcrd + indcrd + valcrd),
                  (long long)ptrcrd, (long long)indcrd, (long long)valcrd, 0);
    head += line;
    std::snprintf(line, sizeof line, "%-14s%14d%14d%14lld%14d\n", "rsa", n, n, (long long)nnz, 0);
    head += line;
    std::snprintf(line, sizeof line, "%-16s%-16s%-20s\n", "(8I10)", "(8I10)", "(4E20.12)");
    head += line;
  }
  Section ps, is, vs;
  ps.count = n + 1, ps.per = ipl, ps.width = iw, ps.start = head.size();
  is.count = nnz, is.per = ipl, is.width = iw, is.start = ps.start + ps.bytes();
  vs.count = nnz, vs.per = vpl, vs.width = vw, vs.start = is.start + is.bytes();
  std::string out(vs.start + vs.bytes(), ' ');
  std::memcpy(&out[0], head.data(), head.size());
  const int nt = nthreads_for(nnz);
  auto fill = [&](const Section& s, auto put) {
    parallel_ranges(s.count, s.count >= 200000 ? nt : 1, [&](int64_t b, int64_t e) {
      for (int64_t i = b; i < e; ++i) {
        char* p = &out[s.at(i)];
        put(p, i);
        if ((i + 1) % s.per == 0 || i + 1 == s.count) p[s.width] = '\n';
      }
    });
  };
  fill(ps, [&](char* p, int64_t i) { put_int(p, iw, (long long)colptr[i]); });
  fill(is, [&](char* p, int64_t i) { put_int(p, iw, (long long)rowind[i]); });
  fill(vs, [&](char* p, int64_t i) {
    char tmp[64];
    const int k = std::snprintf(tmp, sizeof tmp, "%20.12E", nzval[i]);
    if (k <= vw) std::memcpy(p, tmp, vw);
    else std::memcpy(p, tmp + (k - vw), vw);  // cannot happen for finite doubles in E20.12
  });
  FILE* f = std::fopen(path, "wb");
  if (!f) return SPB_ERR_INVALID;
  const size_t wrote = std::fwrite(out.data(), 1, out.size(), f);
  return (std::fclose(f) == 0 && wrote == out.size()) ? SPB_OK : SPB_ERR_INVALID;
}

}  // extern "C"
