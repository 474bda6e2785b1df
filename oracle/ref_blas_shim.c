/*
 * Minimal BLAS/LAPACK entry points for linking the compiled CFFC reference
 * (test infrastructure only; linked into oracle/_ref/e2d_ref_harness and
 * nothing else).
 *
 * The reference's makefile links "-lblas -llapack" with no pinned version
 * (src_2D/makefile.def).  On the Euler2D path it calls:
 *   - BLAS-1 dnrm2/ddot/daxpy/dscal from GMRES
 *     (NewtonKrylovSchwarz2D/GMRES2D.h:546-581, :1029, :1288, :1328, :1434);
 *   - dgetrf/dgetri from BPKIT's dense block inverse used by the block-Jacobi
 *     preconditioner (bpkit/src/DenseMat.h:421-428).
 * These are written here from the published algorithms (reference BLAS
 * scaled 2-norm; LU with partial pivoting, then inversion of U and solution
 * for inv(A) as in LAPACK's unblocked dgetf2/dgetri).  Everything else the
 * link needs is off the Euler2D path and aborts if reached.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

double dnrm2_(const int *n, const double *x, const int *incx) {
  int i, nn = *n, inc = *incx;
  double scale = 0.0, ssq = 1.0;
  if (nn < 1 || inc < 1) return 0.0;
  if (nn == 1) return fabs(x[0]);
  for (i = 0; i < nn; ++i) {
    double v = x[i * inc];
    if (v != 0.0) {
      double a = fabs(v);
      if (scale < a) {
        ssq = 1.0 + ssq * (scale / a) * (scale / a);
        scale = a;
      } else {
        ssq += (a / scale) * (a / scale);
      }
    }
  }
  return scale * sqrt(ssq);
}

double ddot_(const int *n, const double *x, const int *incx, const double *y,
             const int *incy) {
  int i;
  double s = 0.0;
  for (i = 0; i < *n; ++i) s += x[i * *incx] * y[i * *incy];
  return s;
}

void daxpy_(const int *n, const double *a, const double *x, const int *incx,
            double *y, const int *incy) {
  int i;
  if (*a == 0.0) return;
  for (i = 0; i < *n; ++i) y[i * *incy] += *a * x[i * *incx];
}

void dscal_(const int *n, const double *a, double *x, const int *incx) {
  int i;
  for (i = 0; i < *n; ++i) x[i * *incx] *= *a;
}

/* Column-major A(i,j) = a[i + j*lda]. */
#define A_(i, j) a[(i) + (j) * (*lda)]

void dgetrf_(const int *m, const int *n, double *a, const int *lda, int *ipiv,
             int *info) {
  int i, j, k, mn = (*m < *n) ? *m : *n;
  *info = 0;
  for (k = 0; k < mn; ++k) {
    int p = k;
    double amax = fabs(A_(k, k));
    for (i = k + 1; i < *m; ++i)
      if (fabs(A_(i, k)) > amax) { amax = fabs(A_(i, k)); p = i; }
    ipiv[k] = p + 1;
    if (A_(p, k) != 0.0) {
      if (p != k)
        for (j = 0; j < *n; ++j) { double t = A_(k, j); A_(k, j) = A_(p, j); A_(p, j) = t; }
      for (i = k + 1; i < *m; ++i) A_(i, k) /= A_(k, k);
    } else if (*info == 0) {
      *info = k + 1;
    }
    for (j = k + 1; j < *n; ++j)
      for (i = k + 1; i < *m; ++i) A_(i, j) -= A_(i, k) * A_(k, j);
  }
}

void dgetri_(const int *n, double *a, const int *lda, const int *ipiv,
             double *work, const int *lwork, int *info) {
  int i, j, k, nn = *n;
  *info = 0;
  if (*lwork == -1) { work[0] = nn; return; }
  for (k = 0; k < nn; ++k)
    if (A_(k, k) == 0.0) { *info = k + 1; return; }
  /* inv(U) in place (upper triangle). */
  for (j = 0; j < nn; ++j) {
    A_(j, j) = 1.0 / A_(j, j);
    for (i = 0; i < j; ++i) {
      double s = 0.0;
      for (k = i; k < j; ++k) s += A_(i, k) * A_(k, j);
      A_(i, j) = -s * A_(j, j);
    }
  }
  /* Solve inv(A)*L = inv(U) column by column from the right. */
  {
    double *col = (double *)malloc(sizeof(double) * (size_t)nn);
    for (j = nn - 1; j >= 0; --j) {
      for (i = j + 1; i < nn; ++i) { col[i] = A_(i, j); A_(i, j) = 0.0; }
      for (i = 0; i < nn; ++i) {
        double s = A_(i, j);
        for (k = j + 1; k < nn; ++k) s -= A_(i, k) * col[k];
        A_(i, j) = s;
      }
    }
    free(col);
  }
  /* Undo the row interchanges as column interchanges. */
  for (j = nn - 2; j >= 0; --j) {
    int p = ipiv[j] - 1;
    if (p != j)
      for (i = 0; i < nn; ++i) { double t = A_(i, j); A_(i, j) = A_(i, p); A_(i, p) = t; }
  }
}
#undef A_

/* C = alpha*op(A)*op(B) + beta*C, column-major, with the loop order of the
 * reference BLAS (BPKIT's DenseMat products call it for the block-Jacobi
 * preconditioner apply). */
void dgemm_(const char *ta, const char *tb, const int *m, const int *n, const int *k,
            const double *alpha, const double *a, const int *lda, const double *b,
            const int *ldb, const double *beta, double *c, const int *ldc) {
  int i, j, l;
  const int nota = (*ta == 'N' || *ta == 'n'), notb = (*tb == 'N' || *tb == 'n');
#define A(i, j) a[(i) + (j) * (*lda)]
#define B(i, j) b[(i) + (j) * (*ldb)]
#define C(i, j) c[(i) + (j) * (*ldc)]
  if (*m == 0 || *n == 0) return;
  if (*alpha == 0.0) {
    for (j = 0; j < *n; ++j)
      for (i = 0; i < *m; ++i) C(i, j) = (*beta == 0.0) ? 0.0 : *beta * C(i, j);
    return;
  }
  if (notb) {
    if (nota) {
      for (j = 0; j < *n; ++j) {
        if (*beta == 0.0) for (i = 0; i < *m; ++i) C(i, j) = 0.0;
        else if (*beta != 1.0) for (i = 0; i < *m; ++i) C(i, j) = *beta * C(i, j);
        for (l = 0; l < *k; ++l) {
          const double t = *alpha * B(l, j);
          for (i = 0; i < *m; ++i) C(i, j) += t * A(i, l);
        }
      }
    } else {
      for (j = 0; j < *n; ++j)
        for (i = 0; i < *m; ++i) {
          double t = 0.0;
          for (l = 0; l < *k; ++l) t += A(l, i) * B(l, j);
          C(i, j) = (*beta == 0.0) ? *alpha * t : *alpha * t + *beta * C(i, j);
        }
    }
  } else {
    if (nota) {
      for (j = 0; j < *n; ++j) {
        if (*beta == 0.0) for (i = 0; i < *m; ++i) C(i, j) = 0.0;
        else if (*beta != 1.0) for (i = 0; i < *m; ++i) C(i, j) = *beta * C(i, j);
        for (l = 0; l < *k; ++l) {
          const double t = *alpha * B(j, l);
          for (i = 0; i < *m; ++i) C(i, j) += t * A(i, l);
        }
      }
    } else {
      for (j = 0; j < *n; ++j)
        for (i = 0; i < *m; ++i) {
          double t = 0.0;
          for (l = 0; l < *k; ++l) t += A(l, i) * B(j, l);
          C(i, j) = (*beta == 0.0) ? *alpha * t : *alpha * t + *beta * C(i, j);
        }
    }
  }
#undef A
#undef B
#undef C
}

/* Solve A X = B with the LU factors of dgetrf (no transpose only). */
void dgetrs_(const char *tr, const int *n, const int *nrhs, const double *a, const int *lda,
             const int *ipiv, double *b, const int *ldb, int *info) {
  int i, j, k;
  *info = 0;
  if (!(*tr == 'N' || *tr == 'n')) { fprintf(stderr, "dgetrs_: transpose off path\n"); abort(); }
  for (k = 0; k < *nrhs; ++k) {
    double *x = b + k * (*ldb);
    for (i = 0; i < *n; ++i) {
      const int p = ipiv[i] - 1;
      if (p != i) { double t = x[i]; x[i] = x[p]; x[p] = t; }
    }
    for (j = 0; j < *n; ++j)
      for (i = j + 1; i < *n; ++i) x[i] -= x[j] * a[i + j * (*lda)];
    for (j = *n - 1; j >= 0; --j) {
      x[j] /= a[j + j * (*lda)];
      for (i = 0; i < j; ++i) x[i] -= x[j] * a[i + j * (*lda)];
    }
  }
}

static void off_path(const char *name) {
  fprintf(stderr, "e2d_ref_harness: %s is off the Euler2D path and not linked\n", name);
  abort();
}
#define OFF_PATH(sym) void sym(void) { off_path(#sym); }
OFF_PATH(dgesvd_)
OFF_PATH(dgelsy_)
OFF_PATH(dgeev_)
OFF_PATH(dpolft_)
OFF_PATH(dpcoef_)
OFF_PATH(dp1vlu_)
OFF_PATH(bpilut_)
OFF_PATH(bpilutp_)
OFF_PATH(bpilutstat_)
OFF_PATH(bplusol_)
OFF_PATH(readhb_)
OFF_PATH(dgels_)
