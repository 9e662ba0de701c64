/* Part of the GSL-subset shim used only to build the parity oracle: the LU
 * routines PAWAN's resolve.cpp calls (gsl_linalg_LU_decomp / _LU_solve with a
 * gsl_permutation), written here as Gaussian elimination with partial (row)
 * pivoting.  The factors are stored in place, L unit lower triangular below
 * the diagonal and U on and above it, as GSL documents for its LU. */
#ifndef PAWAN_SHIM_GSL_LINALG_H
#define PAWAN_SHIM_GSL_LINALG_H
#include <math.h>
#include <stdlib.h>

#include "pawan_gsl_shim.h"

typedef struct {
  size_t size;
  size_t *data;
} gsl_permutation;

static inline gsl_permutation *gsl_permutation_alloc(const size_t n) {
  gsl_permutation *p = (gsl_permutation *)malloc(sizeof(gsl_permutation));
  if (!p) PAWAN_GSL_FAIL("gsl_permutation_alloc: out of memory");
  p->size = n;
  p->data = (size_t *)malloc((n ? n : 1) * sizeof(size_t));
  if (!p->data) PAWAN_GSL_FAIL("gsl_permutation_alloc: out of memory");
  for (size_t i = 0; i < n; ++i) p->data[i] = i;
  return p;
}

static inline void gsl_permutation_free(gsl_permutation *p) {
  if (!p) return;
  free(p->data);
  free(p);
}

/* A = P^T L U in place; p->data[i] is the original row now at row i. */
static inline int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum) {
  const size_t n = A->size1;
  if (A->size2 != n || p->size != n) PAWAN_GSL_FAIL("gsl_linalg_LU_decomp: needs a square matrix and matching permutation");
  for (size_t i = 0; i < n; ++i) p->data[i] = i;
  int sign = 1;
  for (size_t k = 0; k < n; ++k) {
    size_t piv = k;
    double best = fabs(gsl_matrix_get(A, k, k));
    for (size_t i = k + 1; i < n; ++i) {
      const double v = fabs(gsl_matrix_get(A, i, k));
      if (v > best) { best = v; piv = i; }
    }
    if (piv != k) {
      for (size_t j = 0; j < n; ++j) {
        const double t = gsl_matrix_get(A, k, j);
        gsl_matrix_set(A, k, j, gsl_matrix_get(A, piv, j));
        gsl_matrix_set(A, piv, j, t);
      }
      const size_t t = p->data[k];
      p->data[k] = p->data[piv];
      p->data[piv] = t;
      sign = -sign;
    }
    const double d = gsl_matrix_get(A, k, k);
    if (d == 0.0) continue;  /* singular: left for the solve to report */
    for (size_t i = k + 1; i < n; ++i) {
      const double l = gsl_matrix_get(A, i, k) / d;
      gsl_matrix_set(A, i, k, l);
      for (size_t j = k + 1; j < n; ++j) gsl_matrix_set(A, i, j, gsl_matrix_get(A, i, j) - l * gsl_matrix_get(A, k, j));
    }
  }
  *signum = sign;
  return 0;
}

/* Solves (P^T L U) x = b with the factors of gsl_linalg_LU_decomp. */
static inline int gsl_linalg_LU_solve(const gsl_matrix *LU, const gsl_permutation *p, const gsl_vector *b,
                                      gsl_vector *x) {
  const size_t n = LU->size1;
  if (b->size != n || x->size != n) PAWAN_GSL_FAIL("gsl_linalg_LU_solve: size mismatch");
  double *y = (double *)malloc((n ? n : 1) * sizeof(double));
  if (!y) PAWAN_GSL_FAIL("gsl_linalg_LU_solve: out of memory");
  for (size_t i = 0; i < n; ++i) {
    double s = gsl_vector_get(b, p->data[i]);
    for (size_t j = 0; j < i; ++j) s -= gsl_matrix_get(LU, i, j) * y[j];
    y[i] = s;
  }
  for (size_t ii = n; ii-- > 0;) {
    double s = y[ii];
    for (size_t j = ii + 1; j < n; ++j) s -= gsl_matrix_get(LU, ii, j) * y[j];
    const double d = gsl_matrix_get(LU, ii, ii);
    if (d == 0.0) { free(y); PAWAN_GSL_FAIL("gsl_linalg_LU_solve: singular matrix"); }
    y[ii] = s / d;
  }
  for (size_t i = 0; i < n; ++i) gsl_vector_set(x, i, y[i]);
  free(y);
  return 0;
}

#endif
