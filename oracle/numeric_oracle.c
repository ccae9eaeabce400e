/*
 * ORACLE — test infrastructure only.  Never part of the product path.
 *
 * CPU restatement of symPACK's 2D numeric path at one rank (symPACK v2.0,
 * include/sympack/symPACKMatrix2D.hpp), used as the parity checker of the GPU
 * kernels and as the timed CPU baseline:
 *
 *   cells         one row-major nrows x w_I array per cell (K, I), ld = w_I,
 *                 made of blocks of contiguous rows            2D.hpp:499-944, 3317-3396
 *   distribute    A's lower triangle permuted into the cells   2D.hpp:6336-6576
 *   factorize     Potrf('U', w, diag, w)                        2D.hpp:1052-1102
 *   trsm          Trsm('L','U','T','N', w, m, 1, diag, w, cell, w)  2D.hpp:1104-1178
 *   update        Gemm('T','N', m_J, m_K, w_I) into a buffer, then
 *                 scatter into cell (K, J) through row offsets and
 *                 column indices                               2D.hpp:1180-1469
 *   solve         forward_update(_contrib) / back_update(_contrib)
 *                 with Trsm and Gemm on the permuted RHS       2D.hpp:1486-1797, 5728-6322
 *   get_solution  un-permute                                   2D.hpp:6713-6757
 *
 * LDL^T (DecompositionType::LDL, blockCellLDL_t, 2D.hpp:1802-2465), selected by
 * orc_set_ldl:
 *   factorize     Potrf_LDL('U') of the diagonal cell: unit U = L^T strictly
 *                 above the diagonal, D on it; a zero pivot stops it   lapack.hpp:206-560
 *   trsm          Trsm('L','U','T','U') then column I scaled by 1/D_I   2D.hpp:2118-2137
 *   update        Gemm with W = D L_J^T (computeDLT) instead of L_J^T   2D.hpp:2140-2390
 *   solve         unit forward sweep, scaling by 1/D (scale_contrib), unit
 *                 backward sweep                                        2D.hpp:2392-2462
 *
 * Tasks run in supernode order 1..nsuper, a topological order of the
 * reference's FACTOR -> TRSM -> UPDATE2D_COMP DAG (2D.hpp:3893-3997); at one
 * rank without SP_THREADS the reference also runs them one at a time with a
 * multithreaded BLAS underneath.  The update always takes the general
 * "GEMM into a buffer + scatter" branch; the reference's in-place SYRK/GEMM
 * branch (2D.hpp:1233-1332) computes the same sums.
 *
 * Dense kernels come from scipy's bundled OpenBLAS through its exported
 * scipy_d*_ names (LP64).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

extern void scipy_dpotrf_(const char* uplo, const int* n, double* a, const int* lda, int* info, size_t);
extern void scipy_dtrsm_(const char* side, const char* uplo, const char* transa, const char* diag, const int* m,
                         const int* n, const double* alpha, const double* a, const int* lda, double* b,
                         const int* ldb, size_t, size_t, size_t, size_t);
extern void scipy_dgemm_(const char* ta, const char* tb, const int* m, const int* n, const int* k,
                         const double* alpha, const double* a, const int* lda, const double* b, const int* ldb,
                         const double* beta, double* c, const int* ldc, size_t, size_t);
extern void scipy_openblas_set_num_threads(int);

typedef struct {
  int K;            /* row supernode (1-based) */
  int nrows;
  int nblocks;
  int* blk_first;   /* 1-based first row of each block */
  int* blk_nrows;
  int* blk_off;     /* row offset of each block inside the cell */
  double* nzval;    /* nrows x w_I, row-major */
} cell_t;

typedef struct {
  int n, nsuper;
  int *xsuper, *supmember; /* 1-based */
  int *ncells;             /* per supernode (diagonal cell first) */
  cell_t** cells;          /* per supernode array of cells, K ascending */
  int *invp;               /* 1-based old -> new */
  double* tmp;             /* update buffer */
  size_t tmp_size;
  int status;              /* 0, or the 1-based supernode whose Potrf failed */
  int ldl;                 /* 1: LDL^T (D on the diagonal of the diagonal cells) */
  double* scaled;          /* LDL^T: D-scaled copy of a cell (computeDLT) */
  size_t scaled_size;
} orc_t;

void orc_set_threads(int t) { scipy_openblas_set_num_threads(t); }

static int width(const orc_t* o, int I) { return o->xsuper[I] - o->xsuper[I - 1]; }

/* Cells of every supernode from its row structure: cut where the owning
 * supernode changes, blocks where rows stop being contiguous. */
orc_t* orc_create(int n, int nsuper, const int* xsuper, const int64_t* xlindx, const int* lindx,
                  const int* supmember, const int* invp) {
  orc_t* o = (orc_t*)calloc(1, sizeof(orc_t));
  o->n = n;
  o->nsuper = nsuper;
  o->xsuper = (int*)malloc(sizeof(int) * (nsuper + 1));
  memcpy(o->xsuper, xsuper, sizeof(int) * (nsuper + 1));
  o->supmember = (int*)malloc(sizeof(int) * n);
  memcpy(o->supmember, supmember, sizeof(int) * n);
  o->invp = (int*)malloc(sizeof(int) * n);
  memcpy(o->invp, invp, sizeof(int) * n);
  o->ncells = (int*)calloc(nsuper + 1, sizeof(int));
  o->cells = (cell_t**)calloc(nsuper + 1, sizeof(cell_t*));
  size_t maxrows = 0;
  for (int I = 1; I <= nsuper; ++I) {
    int64_t b = xlindx[I - 1], e = xlindx[I];
    int w = width(o, I);
    if ((size_t)(e - b) > maxrows) maxrows = (size_t)(e - b);
    /* count cells */
    int nc = 0, prevK = -1;
    for (int64_t p = b; p < e; ++p) {
      int K = supmember[lindx[p - 1] - 1];
      if (K != prevK) ++nc;
      prevK = K;
    }
    o->ncells[I] = nc;
    o->cells[I] = (cell_t*)calloc(nc, sizeof(cell_t));
    int ci = -1;
    prevK = -1;
    int prevrow = -2;
    for (int64_t p = b; p < e; ++p) {
      int row = lindx[p - 1];
      int K = supmember[row - 1];
      if (K != prevK) {
        ++ci;
        cell_t* c = &o->cells[I][ci];
        c->K = K;
        /* upper bound on the blocks of this cell */
        int64_t q = p;
        while (q < e && supmember[lindx[q - 1] - 1] == K) ++q;
        int cap = (int)(q - p);
        c->blk_first = (int*)malloc(sizeof(int) * cap);
        c->blk_nrows = (int*)malloc(sizeof(int) * cap);
        c->blk_off = (int*)malloc(sizeof(int) * cap);
        prevrow = -2;
      }
      cell_t* c = &o->cells[I][ci];
      if (row != prevrow + 1) {
        c->blk_first[c->nblocks] = row;
        c->blk_nrows[c->nblocks] = 0;
        c->blk_off[c->nblocks] = c->nrows;
        c->nblocks++;
      }
      c->blk_nrows[c->nblocks - 1]++;
      c->nrows++;
      prevrow = row;
      prevK = K;
    }
    for (int k = 0; k < nc; ++k) o->cells[I][k].nzval = (double*)calloc((size_t)o->cells[I][k].nrows * w, sizeof(double));
  }
  o->tmp_size = maxrows * maxrows;
  o->tmp = (double*)malloc(sizeof(double) * (o->tmp_size ? o->tmp_size : 1));
  return o;
}

void orc_destroy(orc_t* o) {
  if (!o) return;
  for (int I = 1; I <= o->nsuper; ++I) {
    for (int k = 0; k < o->ncells[I]; ++k) {
      cell_t* c = &o->cells[I][k];
      free(c->blk_first);
      free(c->blk_nrows);
      free(c->blk_off);
      free(c->nzval);
    }
    free(o->cells[I]);
  }
  free(o->cells);
  free(o->ncells);
  free(o->xsuper);
  free(o->supmember);
  free(o->invp);
  free(o->tmp);
  free(o->scaled);
  free(o);
}

/* Row offset of global row `row` (1-based) inside a cell, or -1. */
static int cell_row(const cell_t* c, int row) {
  int lo = 0, hi = c->nblocks - 1;
  while (lo <= hi) {
    int mid = (lo + hi) / 2;
    if (row < c->blk_first[mid]) hi = mid - 1;
    else if (row >= c->blk_first[mid] + c->blk_nrows[mid]) lo = mid + 1;
    else return c->blk_off[mid] + (row - c->blk_first[mid]);
  }
  return -1;
}

static cell_t* find_cell(orc_t* o, int I, int K) {
  int lo = 0, hi = o->ncells[I] - 1;
  while (lo <= hi) {
    int mid = (lo + hi) / 2;
    int k = o->cells[I][mid].K;
    if (K < k) hi = mid - 1;
    else if (K > k) lo = mid + 1;
    else return &o->cells[I][mid];
  }
  return NULL;
}

/* DistributeMatrix: (r, c) of A's lower triangle -> permuted (max, min). */
int orc_distribute(orc_t* o, const int64_t* colptr, const int* rowind, const double* nzval) {
  for (int I = 1; I <= o->nsuper; ++I)
    for (int k = 0; k < o->ncells[I]; ++k)
      memset(o->cells[I][k].nzval, 0, sizeof(double) * (size_t)o->cells[I][k].nrows * width(o, I));
  for (int c = 1; c <= o->n; ++c)
    for (int64_t p = colptr[c - 1]; p < colptr[c]; ++p) {
      int r = rowind[p - 1];
      int pr = o->invp[r - 1], pc = o->invp[c - 1];
      if (pr < pc) { int t = pr; pr = pc; pc = t; }
      int I = o->supmember[pc - 1], K = o->supmember[pr - 1];
      cell_t* cl = find_cell(o, I, K);
      if (!cl) return -6;
      int lr = cell_row(cl, pr);
      if (lr < 0) return -6;
      cl->nzval[(size_t)lr * width(o, I) + (pc - o->xsuper[I - 1])] = nzval[p - 1];
    }
  o->status = 0;
  return 0;
}

void orc_set_ldl(orc_t* o, int ldl) { o->ldl = ldl; }

/* Potf2_LDL('U', n, A, lda) (lapack.hpp:206-270): A = U^T D U with unit upper U,
 * column by column; returns the 1-based column of a zero pivot, or 0.  Potrf_LDL
 * (lapack.hpp:398-560) blocks the same recurrence by 64 columns. */
static int potf2_ldl_upper(int n, double* A, int lda, double* work) {
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < j; ++i) work[i] = A[i + (size_t)j * lda] * A[i + (size_t)i * lda];
    double ajj = A[j + (size_t)j * lda];
    for (int i = 0; i < j; ++i) ajj -= A[i + (size_t)j * lda] * work[i];
    A[j + (size_t)j * lda] = ajj;
    if (!(fabs(ajj) > 0)) return j + 1;
    for (int c = j + 1; c < n; ++c) {
      double t = A[j + (size_t)c * lda];
      for (int i = 0; i < j; ++i) t -= A[i + (size_t)c * lda] * work[i];
      A[j + (size_t)c * lda] = t * (1.0 / ajj);
    }
  }
  return 0;
}

static double* scaled_buffer(orc_t* o, size_t need) {
  if (need > o->scaled_size) {
    free(o->scaled);
    o->scaled = (double*)malloc(sizeof(double) * need);
    o->scaled_size = o->scaled ? need : 0;
  }
  return o->scaled;
}

int orc_factorize(orc_t* o) {
  const double one = 1.0, zero = 0.0;
  for (int I = 1; I <= o->nsuper; ++I) {
    int w = width(o, I), info = 0;
    cell_t* diag = &o->cells[I][0];
    /* FACTOR */
    if (o->ldl) {
      double* work = scaled_buffer(o, (size_t)w);
      if (!work) return -3;
      info = potf2_ldl_upper(w, diag->nzval, w, work);
    } else {
      scipy_dpotrf_("U", &w, diag->nzval, &w, &info, 1);
    }
    if (info != 0) {
      o->status = I;
      return -2;
    }
    /* TRSM of every off-diagonal cell */
    for (int k = 1; k < o->ncells[I]; ++k) {
      cell_t* c = &o->cells[I][k];
      scipy_dtrsm_("L", "U", "T", o->ldl ? "U" : "N", &w, &c->nrows, &one, diag->nzval, &w, c->nzval, &w, 1, 1, 1,
                   1);
      if (o->ldl)
        for (int q = 0; q < c->nrows; ++q)
          for (int j = 0; j < w; ++j) c->nzval[(size_t)q * w + j] *= 1.0 / diag->nzval[(size_t)j * w + j];
    }
    /* UPDATE2D_COMP: target (K, J) -= L_KI L_JI^T for K >= J */
    for (int jj = 1; jj < o->ncells[I]; ++jj) {
      cell_t* cj = &o->cells[I][jj];
      int J = cj->K, wJ = width(o, J), fcJ = o->xsuper[J - 1];
      for (int kk = jj; kk < o->ncells[I]; ++kk) {
        cell_t* ck = &o->cells[I][kk];
        int K = ck->K;
        cell_t* tgt = find_cell(o, J, K);
        if (!tgt) return -6;
        int mJ = cj->nrows, mK = ck->nrows;
        /* buf (column-major mJ x mK) = LJ^T-view * LK-view; LDL^T: D LJ^T-view */
        const double* lj = cj->nzval;
        if (o->ldl) {
          double* S = scaled_buffer(o, (size_t)mJ * w);
          if (!S) return -3;
          for (int q = 0; q < mJ; ++q)
            for (int j = 0; j < w; ++j) S[(size_t)q * w + j] = diag->nzval[(size_t)j * w + j] * cj->nzval[(size_t)q * w + j];
          lj = S;
        }
        scipy_dgemm_("T", "N", &mJ, &mK, &w, &one, lj, &w, ck->nzval, &w, &zero, o->tmp, &mJ, 1, 1);
        /* scatter: row k of the K cell -> target row offset, row j of the J cell -> target column */
        int kr = 0;
        for (int b = 0; b < ck->nblocks; ++b)
          for (int q = 0; q < ck->blk_nrows[b]; ++q, ++kr) {
            int grow = ck->blk_first[b] + q;
            int trow = cell_row(tgt, grow);
            if (trow < 0) return -6;
            double* trowp = tgt->nzval + (size_t)trow * wJ;
            const double* src = o->tmp + (size_t)kr * mJ;
            int jr = 0;
            for (int bj = 0; bj < cj->nblocks; ++bj)
              for (int qj = 0; qj < cj->blk_nrows[bj]; ++qj, ++jr) {
                int gcol = cj->blk_first[bj] + qj;
                if (gcol > grow) continue; /* upper part of a diagonal target */
                trowp[gcol - fcJ] -= src[jr];
              }
          }
      }
    }
  }
  return 0;
}

/* Solve in place on B (n x nrhs, column-major, leading dimension ldb, original order). */
int orc_solve(orc_t* o, double* B, int nrhs, int64_t ldb) {
  const int n = o->n;
  const double one = 1.0, mone = -1.0;
  double* Y = (double*)malloc(sizeof(double) * (size_t)n * nrhs);
  if (!Y) return -3;
  for (int c = 0; c < nrhs; ++c)
    for (int i = 0; i < n; ++i) Y[(size_t)(o->invp[i] - 1) + (size_t)c * n] = B[i + c * ldb];
  /* forward: Y_J <- L_JJ^-1 Y_J ; Y_K[rows] -= L_KJ Y_J */
  for (int J = 1; J <= o->nsuper; ++J) {
    int w = width(o, J);
    double* YJ = Y + (o->xsuper[J - 1] - 1);
    scipy_dtrsm_("L", "U", "T", o->ldl ? "U" : "N", &w, &nrhs, &one, o->cells[J][0].nzval, &w, YJ, &n, 1, 1, 1, 1);
    for (int k = 1; k < o->ncells[J]; ++k) {
      cell_t* c = &o->cells[J][k];
      for (int b = 0; b < c->nblocks; ++b) {
        int nr = c->blk_nrows[b];
        scipy_dgemm_("T", "N", &nr, &nrhs, &w, &mone, c->nzval + (size_t)c->blk_off[b] * w, &w, YJ, &n, &one,
                     Y + (c->blk_first[b] - 1), &n, 1, 1);
      }
    }
  }
  /* LDL^T: Y <- D^-1 Y (scale_contrib) */
  if (o->ldl)
    for (int J = 1; J <= o->nsuper; ++J) {
      int w = width(o, J);
      const double* dg = o->cells[J][0].nzval;
      for (int c = 0; c < nrhs; ++c)
        for (int j = 0; j < w; ++j) Y[(size_t)(o->xsuper[J - 1] - 1 + j) + (size_t)c * n] /= dg[(size_t)j * w + j];
    }
  /* backward: X_J -= L_KJ^T X_K[rows] ; X_J <- L_JJ^-T X_J */
  for (int J = o->nsuper; J >= 1; --J) {
    int w = width(o, J);
    double* XJ = Y + (o->xsuper[J - 1] - 1);
    for (int k = 1; k < o->ncells[J]; ++k) {
      cell_t* c = &o->cells[J][k];
      for (int b = 0; b < c->nblocks; ++b) {
        int nr = c->blk_nrows[b];
        scipy_dgemm_("N", "N", &w, &nrhs, &nr, &mone, c->nzval + (size_t)c->blk_off[b] * w, &w,
                     Y + (c->blk_first[b] - 1), &n, &one, XJ, &n, 1, 1);
      }
    }
    scipy_dtrsm_("L", "U", "N", o->ldl ? "U" : "N", &w, &nrhs, &one, o->cells[J][0].nzval, &w, XJ, &n, 1, 1, 1, 1);
  }
  for (int c = 0; c < nrhs; ++c)
    for (int i = 0; i < n; ++i) B[i + c * ldb] = Y[(size_t)(o->invp[i] - 1) + (size_t)c * n];
  free(Y);
  return 0;
}

int orc_status(const orc_t* o) { return o->status; }

/* Factor in the product's dump format: per supernode, h x w column-major with
 * ld h (rows in structure order), entries above the diagonal set to zero. */
void orc_get_factor(const orc_t* o, double* out) {
  size_t pos = 0;
  for (int I = 1; I <= o->nsuper; ++I) {
    int w = width(o, I), h = 0;
    for (int k = 0; k < o->ncells[I]; ++k) h += o->cells[I][k].nrows;
    int r = 0;
    for (int k = 0; k < o->ncells[I]; ++k) {
      const cell_t* c = &o->cells[I][k];
      for (int q = 0; q < c->nrows; ++q, ++r)
        for (int j = 0; j < w; ++j) out[pos + r + (size_t)j * h] = (k == 0 && q < j) ? 0.0 : c->nzval[(size_t)q * w + j];
    }
    pos += (size_t)h * w;
  }
}
