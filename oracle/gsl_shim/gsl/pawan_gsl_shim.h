/*
 * Header-only subset of the GNU Scientific Library interface, written for this
 * project so that PAWAN's own (unmodified) C++ sources can be compiled here as
 * the parity oracle.  GSL itself is not installed in this image and there is no
 * network to fetch it.
 *
 * TEST INFRASTRUCTURE ONLY: nothing on the product path includes this file.
 *
 * Semantics kept from GSL where PAWAN depends on them:
 *   - vectors/matrices are calloc-backed (zero-initialised);
 *   - element get/set are range-checked and abort on a bad index (GSL's default
 *     error handler aborts);
 *   - binary fwrite/fread write the elements as raw doubles;
 *   - dnrm2 uses a scaled sum of squares (the reference-BLAS formulation), so it
 *     neither overflows nor underflows for moderate inputs.
 * Only the symbols the PAWAN sources use are provided (see the symbol list in
 * the PAWAN interaction/integration/wake/system/io sources).  The spline and
 * interpolation entry points exist so wake.cpp links; they abort if called,
 * because the Dymore-coupling code that uses them is not exercised.
 */
#ifndef PAWAN_GSL_SHIM_H_
#define PAWAN_GSL_SHIM_H_

#include <float.h> /* GSL's gsl_math.h pulls this in through gsl_machine.h */
#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---------------------------------------------------------------- errors */
static inline void pawan_gsl_fail(const char *what, const char *file, int line) {
  fprintf(stderr, "gsl shim: %s (%s:%d)\n", what, file, line);
  abort();
}
#define PAWAN_GSL_FAIL(msg) pawan_gsl_fail(msg, __FILE__, __LINE__)

/* ---------------------------------------------------------------- math */
static inline double gsl_pow_2(const double x) { return x * x; }
static inline double gsl_pow_3(const double x) { return x * x * x; }
static inline double gsl_pow_4(const double x) { double x2 = x * x; return x2 * x2; }
static inline double gsl_pow_7(const double x) { double x2 = x * x; double x4 = x2 * x2; return x4 * x2 * x; }
static inline double gsl_hypot(const double x, const double y) { return hypot(x, y); }
static inline double gsl_hypot3(const double x, const double y, const double z) {
  double ax = fabs(x), ay = fabs(y), az = fabs(z);
  double m = ax > ay ? (ax > az ? ax : az) : (ay > az ? ay : az);
  if (m == 0.0) return 0.0;
  double rx = ax / m, ry = ay / m, rz = az / m;
  return m * sqrt(rx * rx + ry * ry + rz * rz);
}

/* ---------------------------------------------------------------- block */
typedef struct { size_t size; double *data; } gsl_block;

/* ---------------------------------------------------------------- vector */
typedef struct {
  size_t size;
  size_t stride;
  double *data;
  gsl_block *block;
  int owner;
} gsl_vector;

typedef struct { gsl_vector vector; } _gsl_vector_view;
typedef _gsl_vector_view gsl_vector_view;
typedef struct { gsl_vector vector; } _gsl_vector_const_view;
typedef const _gsl_vector_const_view gsl_vector_const_view;

static inline gsl_vector *gsl_vector_calloc(const size_t n) {
  gsl_vector *v = (gsl_vector *)malloc(sizeof(gsl_vector));
  gsl_block *b = (gsl_block *)malloc(sizeof(gsl_block));
  if (!v || !b) PAWAN_GSL_FAIL("out of memory");
  b->size = n;
  b->data = (double *)calloc(n ? n : 1, sizeof(double));
  if (!b->data) PAWAN_GSL_FAIL("out of memory");
  v->size = n; v->stride = 1; v->data = b->data; v->block = b; v->owner = 1;
  return v;
}
static inline gsl_vector *gsl_vector_alloc(const size_t n) { return gsl_vector_calloc(n); }
static inline void gsl_vector_free(gsl_vector *v) {
  if (!v) return;
  if (v->owner) { free(v->block->data); free(v->block); }
  free(v);
}
static inline double gsl_vector_get(const gsl_vector *v, const size_t i) {
  if (i >= v->size) PAWAN_GSL_FAIL("vector index out of range");
  return v->data[i * v->stride];
}
static inline void gsl_vector_set(gsl_vector *v, const size_t i, double x) {
  if (i >= v->size) PAWAN_GSL_FAIL("vector index out of range");
  v->data[i * v->stride] = x;
}
static inline double *gsl_vector_ptr(gsl_vector *v, const size_t i) {
  if (i >= v->size) PAWAN_GSL_FAIL("vector index out of range");
  return v->data + i * v->stride;
}
static inline void gsl_vector_set_zero(gsl_vector *v) {
  for (size_t i = 0; i < v->size; ++i) v->data[i * v->stride] = 0.0;
}
static inline void gsl_vector_set_all(gsl_vector *v, double x) {
  for (size_t i = 0; i < v->size; ++i) v->data[i * v->stride] = x;
}
static inline int gsl_vector_memcpy(gsl_vector *dst, const gsl_vector *src) {
  if (dst->size != src->size) PAWAN_GSL_FAIL("vector lengths are not equal");
  for (size_t i = 0; i < src->size; ++i) dst->data[i * dst->stride] = src->data[i * src->stride];
  return 0;
}
static inline int gsl_vector_add(gsl_vector *a, const gsl_vector *b) {
  if (a->size != b->size) PAWAN_GSL_FAIL("vector lengths are not equal");
  for (size_t i = 0; i < a->size; ++i) a->data[i * a->stride] += b->data[i * b->stride];
  return 0;
}
static inline int gsl_vector_sub(gsl_vector *a, const gsl_vector *b) {
  if (a->size != b->size) PAWAN_GSL_FAIL("vector lengths are not equal");
  for (size_t i = 0; i < a->size; ++i) a->data[i * a->stride] -= b->data[i * b->stride];
  return 0;
}
static inline int gsl_vector_scale(gsl_vector *a, const double x) {
  for (size_t i = 0; i < a->size; ++i) a->data[i * a->stride] *= x;
  return 0;
}
static inline _gsl_vector_view gsl_vector_subvector(gsl_vector *v, size_t offset, size_t n) {
  if (offset + n > v->size) PAWAN_GSL_FAIL("subvector out of range");
  _gsl_vector_view view;
  view.vector.size = n; view.vector.stride = v->stride;
  view.vector.data = v->data + offset * v->stride;
  view.vector.block = v->block; view.vector.owner = 0;
  return view;
}
static inline _gsl_vector_const_view gsl_vector_const_subvector(const gsl_vector *v, size_t offset, size_t n) {
  if (offset + n > v->size) PAWAN_GSL_FAIL("subvector out of range");
  _gsl_vector_const_view view;
  view.vector.size = n; view.vector.stride = v->stride;
  view.vector.data = v->data + offset * v->stride;
  view.vector.block = v->block; view.vector.owner = 0;
  return view;
}
static inline int gsl_vector_fwrite(FILE *f, const gsl_vector *v) {
  for (size_t i = 0; i < v->size; ++i)
    if (fwrite(v->data + i * v->stride, sizeof(double), 1, f) != 1) return 1;
  return 0;
}
static inline int gsl_vector_fread(FILE *f, gsl_vector *v) {
  for (size_t i = 0; i < v->size; ++i)
    if (fread(v->data + i * v->stride, sizeof(double), 1, f) != 1) return 1;
  return 0;
}

/* ---------------------------------------------------------------- matrix */
typedef struct {
  size_t size1;
  size_t size2;
  size_t tda;
  double *data;
  gsl_block *block;
  int owner;
} gsl_matrix;

typedef struct { gsl_matrix matrix; } _gsl_matrix_view;
typedef _gsl_matrix_view gsl_matrix_view;
typedef struct { gsl_matrix matrix; } _gsl_matrix_const_view;
typedef const _gsl_matrix_const_view gsl_matrix_const_view;

static inline gsl_matrix *gsl_matrix_calloc(const size_t n1, const size_t n2) {
  gsl_matrix *m = (gsl_matrix *)malloc(sizeof(gsl_matrix));
  gsl_block *b = (gsl_block *)malloc(sizeof(gsl_block));
  if (!m || !b) PAWAN_GSL_FAIL("out of memory");
  b->size = n1 * n2;
  b->data = (double *)calloc(b->size ? b->size : 1, sizeof(double));
  if (!b->data) PAWAN_GSL_FAIL("out of memory");
  m->size1 = n1; m->size2 = n2; m->tda = n2; m->data = b->data; m->block = b; m->owner = 1;
  return m;
}
static inline gsl_matrix *gsl_matrix_alloc(const size_t n1, const size_t n2) { return gsl_matrix_calloc(n1, n2); }
static inline void gsl_matrix_free(gsl_matrix *m) {
  if (!m) return;
  if (m->owner) { free(m->block->data); free(m->block); }
  free(m);
}
static inline double gsl_matrix_get(const gsl_matrix *m, const size_t i, const size_t j) {
  if (i >= m->size1 || j >= m->size2) PAWAN_GSL_FAIL("matrix index out of range");
  return m->data[i * m->tda + j];
}
static inline void gsl_matrix_set(gsl_matrix *m, const size_t i, const size_t j, const double x) {
  if (i >= m->size1 || j >= m->size2) PAWAN_GSL_FAIL("matrix index out of range");
  m->data[i * m->tda + j] = x;
}
static inline void gsl_matrix_set_zero(gsl_matrix *m) {
  for (size_t i = 0; i < m->size1; ++i)
    for (size_t j = 0; j < m->size2; ++j) m->data[i * m->tda + j] = 0.0;
}
static inline int gsl_matrix_memcpy(gsl_matrix *dst, const gsl_matrix *src) {
  if (dst->size1 != src->size1 || dst->size2 != src->size2) PAWAN_GSL_FAIL("matrix sizes are different");
  for (size_t i = 0; i < src->size1; ++i)
    for (size_t j = 0; j < src->size2; ++j) dst->data[i * dst->tda + j] = src->data[i * src->tda + j];
  return 0;
}
static inline _gsl_vector_view gsl_matrix_row(gsl_matrix *m, const size_t i) {
  if (i >= m->size1) PAWAN_GSL_FAIL("row index out of range");
  _gsl_vector_view view;
  view.vector.size = m->size2; view.vector.stride = 1;
  view.vector.data = m->data + i * m->tda; view.vector.block = m->block; view.vector.owner = 0;
  return view;
}
static inline _gsl_vector_const_view gsl_matrix_const_row(const gsl_matrix *m, const size_t i) {
  if (i >= m->size1) PAWAN_GSL_FAIL("row index out of range");
  _gsl_vector_const_view view;
  view.vector.size = m->size2; view.vector.stride = 1;
  view.vector.data = m->data + i * m->tda; view.vector.block = m->block; view.vector.owner = 0;
  return view;
}
static inline _gsl_vector_view gsl_matrix_column(gsl_matrix *m, const size_t j) {
  if (j >= m->size2) PAWAN_GSL_FAIL("column index out of range");
  _gsl_vector_view view;
  view.vector.size = m->size1; view.vector.stride = m->tda;
  view.vector.data = m->data + j; view.vector.block = m->block; view.vector.owner = 0;
  return view;
}
static inline _gsl_matrix_const_view gsl_matrix_const_view_vector(const gsl_vector *v, const size_t n1, const size_t n2) {
  if (v->stride != 1) PAWAN_GSL_FAIL("vector must have unit stride");
  if (n1 * n2 > v->size) PAWAN_GSL_FAIL("matrix size exceeds size of original");
  _gsl_matrix_const_view view;
  view.matrix.size1 = n1; view.matrix.size2 = n2; view.matrix.tda = n2;
  view.matrix.data = v->data; view.matrix.block = v->block; view.matrix.owner = 0;
  return view;
}
static inline _gsl_matrix_view gsl_matrix_view_vector(gsl_vector *v, const size_t n1, const size_t n2) {
  if (v->stride != 1) PAWAN_GSL_FAIL("vector must have unit stride");
  if (n1 * n2 > v->size) PAWAN_GSL_FAIL("matrix size exceeds size of original");
  _gsl_matrix_view view;
  view.matrix.size1 = n1; view.matrix.size2 = n2; view.matrix.tda = n2;
  view.matrix.data = v->data; view.matrix.block = v->block; view.matrix.owner = 0;
  return view;
}
static inline int gsl_matrix_fwrite(FILE *f, const gsl_matrix *m) {
  for (size_t i = 0; i < m->size1; ++i)
    if (fwrite(m->data + i * m->tda, sizeof(double), m->size2, f) != m->size2) return 1;
  return 0;
}
static inline int gsl_matrix_fread(FILE *f, gsl_matrix *m) {
  for (size_t i = 0; i < m->size1; ++i)
    if (fread(m->data + i * m->tda, sizeof(double), m->size2, f) != m->size2) return 1;
  return 0;
}

/* ---------------------------------------------------------------- BLAS-1/3 */
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_TRANSPOSE CBLAS_TRANSPOSE_t;

static inline int gsl_blas_ddot(const gsl_vector *x, const gsl_vector *y, double *result) {
  if (x->size != y->size) PAWAN_GSL_FAIL("invalid length");
  double r = 0.0;
  for (size_t i = 0; i < x->size; ++i) r += x->data[i * x->stride] * y->data[i * y->stride];
  *result = r;
  return 0;
}
/* Euclidean norm by the scaled sum-of-squares recurrence: keep a running scale
 * (largest magnitude so far) and the sum of squares of the elements divided by
 * that scale. */
static inline double gsl_blas_dnrm2(const gsl_vector *x) {
  const size_t n = x->size;
  if (n == 0) return 0.0;
  if (n == 1) return fabs(x->data[0]);
  double scale = 0.0, ssq = 1.0;
  for (size_t i = 0; i < n; ++i) {
    const double xi = x->data[i * x->stride];
    if (xi != 0.0) {
      const double ax = fabs(xi);
      if (scale < ax) {
        ssq = 1.0 + ssq * (scale / ax) * (scale / ax);
        scale = ax;
      } else {
        ssq += (ax / scale) * (ax / scale);
      }
    }
  }
  return scale * sqrt(ssq);
}
static inline void gsl_blas_dscal(const double alpha, gsl_vector *x) {
  for (size_t i = 0; i < x->size; ++i) x->data[i * x->stride] *= alpha;
}
static inline int gsl_blas_dgemm(CBLAS_TRANSPOSE_t ta, CBLAS_TRANSPOSE_t tb, double alpha,
                                 const gsl_matrix *A, const gsl_matrix *B, double beta, gsl_matrix *C) {
  const size_t M = C->size1, N = C->size2;
  const size_t K = (ta == CblasNoTrans) ? A->size2 : A->size1;
  for (size_t i = 0; i < M; ++i)
    for (size_t j = 0; j < N; ++j) {
      double s = 0.0;
      for (size_t k = 0; k < K; ++k) {
        double a = (ta == CblasNoTrans) ? A->data[i * A->tda + k] : A->data[k * A->tda + i];
        double b = (tb == CblasNoTrans) ? B->data[k * B->tda + j] : B->data[j * B->tda + k];
        s += a * b;
      }
      C->data[i * C->tda + j] = alpha * s + beta * C->data[i * C->tda + j];
    }
  return 0;
}

/* ---------------------------------------------------------------- interpolation (link-only) */
typedef struct { int unused; } gsl_interp_type;
typedef struct { int unused; } gsl_interp_accel;
typedef struct { int unused; } gsl_interp;
typedef struct { int unused; } gsl_spline;
static const gsl_interp_type pawan_gsl_cspline_type = {0};
#define gsl_interp_cspline (&pawan_gsl_cspline_type)
static inline gsl_interp_accel *gsl_interp_accel_alloc(void) { PAWAN_GSL_FAIL("interpolation is not provided by the shim"); return 0; }
static inline void gsl_interp_accel_free(gsl_interp_accel *) { PAWAN_GSL_FAIL("interpolation is not provided by the shim"); }
static inline gsl_spline *gsl_spline_alloc(const gsl_interp_type *, size_t) { PAWAN_GSL_FAIL("interpolation is not provided by the shim"); return 0; }
static inline int gsl_spline_init(gsl_spline *, const double *, const double *, size_t) { PAWAN_GSL_FAIL("interpolation is not provided by the shim"); return 0; }
static inline double gsl_spline_eval(const gsl_spline *, double, gsl_interp_accel *) { PAWAN_GSL_FAIL("interpolation is not provided by the shim"); return 0; }
static inline void gsl_spline_free(gsl_spline *) { PAWAN_GSL_FAIL("interpolation is not provided by the shim"); }

#endif
