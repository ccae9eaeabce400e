"""The C boundary from C: include/sympack_b200.h compiles as C99 and a C program linked
against the library runs the host-only analysis (no GPU needed) and reads the same
results the Python binding reports."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from sympack_b200 import DistSparseMatrix, generators as G, symPACKMatrix2D, symPACKOptions
from sympack_b200.solver import matlab_sparse
from sympack_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include "sympack_b200.h"

/* 2D 5-point Laplacian k x k, lower triangle, 1-based CSC */
int main(int argc, char** argv) {
  const int k = atoi(argv[1]), n = k * k;
  int64_t* colptr = malloc(sizeof(int64_t) * (n + 1));
  int32_t* rowind = malloc(sizeof(int32_t) * 3 * n);
  int64_t nz = 0;
  for (int c = 0; c < n; ++c) {
    colptr[c] = nz + 1;
    rowind[nz++] = c + 1;
    if ((c + 1) % k) rowind[nz++] = c + 2;
    if (c + k < n) rowind[nz++] = c + k + 1;
  }
  colptr[n] = nz + 1;
  spb_options o;
  spb_default_options(&o);
  o.device = -1;                 /* host-only: symbolic analysis */
  o.ordering = SPB_ORDERING_AMD;
  spb_handle* h = NULL;
  if (spb_create(&o, &h) != SPB_OK) return 2;
  int rc = spb_symbolic(h, n, colptr, rowind);
  if (rc != SPB_OK) { fprintf(stderr, "%s\n", spb_last_error(h)); return 3; }
  spb_info info;
  if (spb_get_info(h, &info) != SPB_OK) return 4;
  int32_t* perm = malloc(sizeof(int32_t) * n);
  int32_t* invp = malloc(sizeof(int32_t) * n);
  if (spb_get_ordering(h, perm, invp) != SPB_OK) return 5;
  long long check = 0;
  for (int i = 0; i < n; ++i) check += (long long)(i + 1) * invp[i];
  printf("%d %d %lld %.1f %lld\n", info.n, info.nsuper, (long long)info.nnz_l, info.flops_stat, check);
  /* a device call on a host-only handle is refused, not crashed */
  if (spb_factorize(h) == SPB_OK) return 6;
  spb_destroy(h);
  free(colptr); free(rowind); free(perm); free(invp);
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_program_against_the_library(tmp_path):
    lib = N.load()  # builds the library if needed
    libdir = os.path.dirname(lib._name)
    src = tmp_path / "prog.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "prog"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lsympack_b200", f"-Wl,-rpath,{libdir}"], check=True)
    env = dict(os.environ)
    import nvidia.cuda_runtime as cr  # the CUDA runtime the library links against
    rt = os.path.join(os.path.dirname(cr.__file__), "lib")
    env["LD_LIBRARY_PATH"] = rt + os.pathsep + env.get("LD_LIBRARY_PATH", "")
    out = subprocess.run([str(exe), "24"], check=True, capture_output=True, text=True, env=env).stdout.split()
    n, cp, ri, v = G.laplacian_2d(24, 24)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1, orderingStr="AMD"))
    M.SymbolicFactorization(DistSparseMatrix.from_lower_csc(n, cp, ri, v))
    inf = M.info()
    _, invp = M.GetOrdering()
    assert int(out[0]) == n and int(out[1]) == inf.nsuper and int(out[2]) == inf.nnz_l
    assert float(out[3]) == pytest.approx(inf.flops_stat)
    assert int(out[4]) == int(np.sum(np.arange(1, n + 1, dtype=np.int64) * invp))


CPP_PROGRAM = r"""
#include <cstdio>
#include <fstream>
#include <vector>
#include "sympack_b200.hpp"

// the members of symPACK's DistSparseMatrix<double> at one rank that the class reads
struct Graph { std::vector<long long> colptr; std::vector<int> rowind; };
struct DistSparseMatrix { int size; Graph Localg_; std::vector<double> nzvalLocal; };

int main(int argc, char** argv) {
  const int k = 20, n = k * k;
  DistSparseMatrix A;
  A.size = n;
  for (int c = 0; c < n; ++c) {
    A.Localg_.colptr.push_back((long long)A.Localg_.rowind.size() + 1);
    A.Localg_.rowind.push_back(c + 1); A.nzvalLocal.push_back(4.0);
    if ((c + 1) % k) { A.Localg_.rowind.push_back(c + 2); A.nzvalLocal.push_back(-1.0); }
    if (c + k < n) { A.Localg_.rowind.push_back(c + k + 1); A.nzvalLocal.push_back(-1.0); }
  }
  A.Localg_.colptr.push_back((long long)A.Localg_.rowind.size() + 1);
  // options set the way run_sympack2D sets the reference's symPACKOptions
  sympack_b200::symPACKOptions optionsFact;
  optionsFact.orderingStr = "MMD";
  optionsFact.relax.SetMaxSize(0);
  optionsFact.decomposition = sympack_b200::DecompositionType::LL;
  optionsFact.device = -1;
  sympack_b200::symPACKMatrix2D M;
  M.Init(optionsFact);
  M.SymbolicFactorization(A);
  bool bad_ordering = false;
  sympack_b200::symPACKOptions bad;
  bad.orderingStr = "SCOTCH";
  try { sympack_b200::symPACKMatrix2D B; B.Init(bad); } catch (const std::logic_error&) { bad_ordering = true; }
  std::vector<int> invp;
  std::vector<int> perm = M.GetOrdering(&invp);
  std::vector<int> xsuper = M.GetSupernodalPartition();
  std::vector<int> parent = M.GetETree();
  long long check = 0;
  for (int i = 0; i < n; ++i) check += (long long)(i + 1) * invp[i];
  std::printf("%d %zu %lld %d\n", M.info().nsuper, xsuper.size(), check, parent[n - 1]);
  bool threw = false;
  try { M.Factorize(); } catch (const std::runtime_error&) { threw = true; }  // host-only handle
  std::printf("%d %d\n", threw ? 1 : 0, bad_ordering ? 1 : 0);
  // default options: the reference constructor's supernode cap of 150 columns, lifted
  // by SetMaxSize(0); a dense 300 x 300 matrix is one supernode without the cap
  const int nd = 300;
  std::vector<long long> dcp(1, 1);
  std::vector<int> dri;
  for (int c = 0; c < nd; ++c) {
    for (int r = c; r < nd; ++r) dri.push_back(r + 1);
    dcp.push_back((long long)dri.size() + 1);
  }
  for (int cap = 0; cap < 2; ++cap) {
    sympack_b200::symPACKOptions od;
    od.device = -1;
    if (cap) std::printf("%d %d %d %d ", od.relax.maxSize, od.relax.nrelax0, od.relax.nrelax1, od.relax.nrelax2);
    else od.relax.SetMaxSize(0);
    sympack_b200::symPACKMatrix2D D;
    D.Init(od);
    D.SymbolicFactorization(nd, reinterpret_cast<const int64_t*>(dcp.data()), dri.data());
    std::vector<int> xs = D.GetSupernodalPartition();
    int widest = 0;
    for (size_t s = 0; s + 1 < xs.size(); ++s) widest = std::max(widest, xs[s + 1] - xs[s]);
    std::printf("%d\n", widest);
  }
  // accessors, and the MATLAB text of a made-up factor (value = 1000 row + column)
  std::printf("%d %d %d\n", M.Size(), M.TotalSupernodeCnt(), M.GetOptions().relax.maxSize);
  const spb_info inf = M.info();
  std::vector<int64_t> xl(inf.nsuper + 1);
  std::vector<int32_t> li(inf.lindx_size);
  if (spb_get_structure(M.handle(), xl.data(), li.data()) != SPB_OK) return 1;
  std::vector<double> panels;
  for (int s = 0; s < inf.nsuper; ++s)
    for (int j = xsuper[s]; j < xsuper[s + 1]; ++j)
      for (int64_t i = xl[s] - 1; i < xl[s + 1] - 1; ++i) panels.push_back(1000.0 * li[i] + j);
  std::ofstream out(argv[argc - 1]);
  sympack_b200::write_matlab_sparse(out, n, xsuper, xl, li, panels.data());
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cpp_class_over_the_library(tmp_path):
    lib = N.load()
    libdir = os.path.dirname(lib._name)
    src = tmp_path / "prog.cpp"
    src.write_text(CPP_PROGRAM)
    exe = tmp_path / "progxx"
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe), "-L", libdir, "-lsympack_b200", f"-Wl,-rpath,{libdir}"], check=True)
    import nvidia.cuda_runtime as cr
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = os.path.join(os.path.dirname(cr.__file__), "lib") + os.pathsep + env.get(
        "LD_LIBRARY_PATH", "")
    dump = tmp_path / "L.m"
    out = subprocess.run([str(exe), str(dump)], check=True, capture_output=True, text=True, env=env).stdout.split()
    n, cp, ri, v = G.laplacian_2d(20, 20)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1))
    M.SymbolicFactorization(DistSparseMatrix.from_lower_csc(n, cp, ri, v))
    _, invp = M.GetOrdering()
    assert int(out[0]) == M.info().nsuper and int(out[1]) == M.info().nsuper + 1
    assert int(out[2]) == int(np.sum(np.arange(1, n + 1, dtype=np.int64) * invp))
    assert int(out[3]) == M.GetETree()[-1]
    assert out[4] == "1"
    assert out[5] == "1"  # an ordering the solver does not have is a logic_error, as in the reference
    assert int(out[6]) == 300  # relax.SetMaxSize(0): no cap, the dense block is one supernode
    assert out[7:11] == ["150", "8", "32", "64"]  # symPACKOptions() defaults (Types.hpp:158-188)
    assert int(out[11]) == 150  # ... which cap supernodes at 150 columns
    assert [int(x) for x in out[12:15]] == [n, M.info().nsuper, 0]  # Size, TotalSupernodeCnt, GetOptions
    # DumpMatlab's text: the same as the Python class writes for the same panels
    xs = M.GetSupernodalPartition()
    xl, li = M.GetStructure()
    panels = np.concatenate([(1000.0 * li[xl[s] - 1:xl[s + 1] - 1][:, None]
                              + np.arange(xs[s], xs[s + 1])[None, :]).T.ravel() for s in range(len(xs) - 1)])
    assert dump.read_text() == matlab_sparse(n, xs, xl, li, panels)


CPP_DEVICE_PROGRAM = r"""
#include <cmath>
#include <cstdio>
#include <vector>
#include "sympack_b200.hpp"

struct Graph { std::vector<long long> colptr; std::vector<int> rowind; };
struct DistSparseMatrix { int size; Graph Localg_; std::vector<double> nzvalLocal; };

int main() {
  const int k = 40, n = k * k, nrhs = 3;
  DistSparseMatrix A;
  A.size = n;
  for (int c = 0; c < n; ++c) {
    A.Localg_.colptr.push_back((long long)A.Localg_.rowind.size() + 1);
    A.Localg_.rowind.push_back(c + 1); A.nzvalLocal.push_back(4.01);
    if ((c + 1) % k) { A.Localg_.rowind.push_back(c + 2); A.nzvalLocal.push_back(-1.0); }
    if (c + k < n) { A.Localg_.rowind.push_back(c + k + 1); A.nzvalLocal.push_back(-1.0); }
  }
  A.Localg_.colptr.push_back((long long)A.Localg_.rowind.size() + 1);
  std::vector<double> b(n * nrhs), x(n * nrhs, 0.0);
  for (int i = 0; i < n * nrhs; ++i) b[i] = std::sin(0.37 * i);
  sympack_b200::symPACKOptions optionsFact;  // device 0, FP64, MMD
  sympack_b200::symPACKMatrix2D M;
  M.Init(optionsFact);
  M.SymbolicFactorization(A);
  M.DistributeMatrix(A);
  M.Factorize();
  M.Solve(b.data(), nrhs, n, nullptr);  // symPACKMatrixMeta::Solve(RHS, nrhs, rhs_size, Xptr)
  M.GetSolution(x.data(), nrhs);
  // residual ||A x - b|| / ||b|| with the symmetric matrix from its lower triangle
  double rn = 0.0, bn = 0.0;
  for (int c = 0; c < nrhs; ++c) {
    std::vector<double> r(b.begin() + c * n, b.begin() + (c + 1) * n);
    for (int j = 0; j < n; ++j)
      for (long long p = A.Localg_.colptr[j] - 1; p < A.Localg_.colptr[j + 1] - 1; ++p) {
        const int i = A.Localg_.rowind[p] - 1;
        const double v = A.nzvalLocal[p];
        r[i] -= v * x[c * n + j];
        if (i != j) r[j] -= v * x[c * n + i];
      }
    for (int i = 0; i < n; ++i) { rn += r[i] * r[i]; bn += b[c * n + i] * b[c * n + i]; }
  }
  std::printf("%.3e\n", std::sqrt(rn / bn));
  return 0;
}
"""


@pytest.mark.gpu
def test_cpp_class_factor_and_solve_on_the_device(tmp_path):
    lib = N.load()
    libdir = os.path.dirname(lib._name)
    src = tmp_path / "dev.cpp"
    src.write_text(CPP_DEVICE_PROGRAM)
    exe = tmp_path / "devxx"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe), "-L",
                    libdir, "-lsympack_b200", f"-Wl,-rpath,{libdir}"], check=True)
    import nvidia.cuda_runtime as cr
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = os.path.join(os.path.dirname(cr.__file__), "lib") + os.pathsep + env.get(
        "LD_LIBRARY_PATH", "")
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, env=env, timeout=300).stdout
    assert float(out.split()[0]) < 1e-13
