/* Test infrastructure: implementation of the GSL-API subset declared in
 * gsl/*.h.  Written for this project from the public GSL API documentation;
 * it exists only so that the reference's unmodified C++ sources can be compiled
 * here and used as the parity oracle and as the timed CPU baseline.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gsl/gsl_blas.h"
#include "gsl/gsl_linalg.h"
#include "gsl/gsl_math.h"
#include "gsl/gsl_matrix.h"
#include "gsl/gsl_permutation.h"
#include "gsl/gsl_vector.h"

void gslshim_fail(const char *what, const char *file, int line) {
  fprintf(stderr, "gsl shim: %s (%s:%d)\n", what, file, line);
  abort();
}

#define SHIM_REQUIRE(cond, msg) \
  do {                          \
    if (!(cond)) gslshim_fail(msg, __FILE__, __LINE__); \
  } while (0)

/* ---------------------------------------------------------------- blocks */

static gsl_block *block_alloc(size_t n, int zero) {
  gsl_block *b = (gsl_block *)malloc(sizeof(gsl_block));
  SHIM_REQUIRE(b != NULL, "block struct allocation failed");
  b->data = zero ? (double *)calloc(n ? n : 1, sizeof(double))
                 : (double *)malloc((n ? n : 1) * sizeof(double));
  SHIM_REQUIRE(b->data != NULL, "block data allocation failed");
  b->size = n;
  return b;
}

static void block_free(gsl_block *b) {
  if (!b) return;
  free(b->data);
  free(b);
}

/* --------------------------------------------------------------- vectors */

static gsl_vector *vector_make(size_t n, int zero) {
  gsl_vector *v = (gsl_vector *)malloc(sizeof(gsl_vector));
  SHIM_REQUIRE(v != NULL, "vector struct allocation failed");
  v->block = block_alloc(n, zero);
  v->data = v->block->data;
  v->size = n;
  v->stride = 1;
  v->owner = 1;
  return v;
}

gsl_vector *gsl_vector_alloc(size_t n) { return vector_make(n, 0); }
gsl_vector *gsl_vector_calloc(size_t n) { return vector_make(n, 1); }

void gsl_vector_free(gsl_vector *v) {
  if (!v) return;
  if (v->owner) block_free(v->block);
  free(v);
}

double gsl_vector_get(const gsl_vector *v, size_t i) {
  SHIM_REQUIRE(i < v->size, "vector index out of range");
  return v->data[i * v->stride];
}

void gsl_vector_set(gsl_vector *v, size_t i, double x) {
  SHIM_REQUIRE(i < v->size, "vector index out of range");
  v->data[i * v->stride] = x;
}

double *gsl_vector_ptr(gsl_vector *v, size_t i) {
  SHIM_REQUIRE(i < v->size, "vector index out of range");
  return v->data + i * v->stride;
}

void gsl_vector_set_zero(gsl_vector *v) {
  for (size_t i = 0; i < v->size; ++i) v->data[i * v->stride] = 0.0;
}

void gsl_vector_set_all(gsl_vector *v, double x) {
  for (size_t i = 0; i < v->size; ++i) v->data[i * v->stride] = x;
}

int gsl_vector_memcpy(gsl_vector *dest, const gsl_vector *src) {
  SHIM_REQUIRE(dest->size == src->size, "vector lengths differ in memcpy");
  for (size_t i = 0; i < src->size; ++i)
    dest->data[i * dest->stride] = src->data[i * src->stride];
  return GSL_SUCCESS;
}

int gsl_vector_add(gsl_vector *a, const gsl_vector *b) {
  SHIM_REQUIRE(a->size == b->size, "vector lengths differ in add");
  for (size_t i = 0; i < a->size; ++i) a->data[i * a->stride] += b->data[i * b->stride];
  return GSL_SUCCESS;
}

int gsl_vector_sub(gsl_vector *a, const gsl_vector *b) {
  SHIM_REQUIRE(a->size == b->size, "vector lengths differ in sub");
  for (size_t i = 0; i < a->size; ++i) a->data[i * a->stride] -= b->data[i * b->stride];
  return GSL_SUCCESS;
}

int gsl_vector_mul(gsl_vector *a, const gsl_vector *b) {
  SHIM_REQUIRE(a->size == b->size, "vector lengths differ in mul");
  for (size_t i = 0; i < a->size; ++i) a->data[i * a->stride] *= b->data[i * b->stride];
  return GSL_SUCCESS;
}

int gsl_vector_scale(gsl_vector *a, double x) {
  for (size_t i = 0; i < a->size; ++i) a->data[i * a->stride] *= x;
  return GSL_SUCCESS;
}

int gsl_vector_add_constant(gsl_vector *a, double x) {
  for (size_t i = 0; i < a->size; ++i) a->data[i * a->stride] += x;
  return GSL_SUCCESS;
}

gsl_vector_view gsl_vector_subvector(gsl_vector *v, size_t offset, size_t n) {
  SHIM_REQUIRE(offset + n <= v->size, "subvector out of range");
  gsl_vector_view view;
  view.vector.size = n;
  view.vector.stride = v->stride;
  view.vector.data = v->data + offset * v->stride;
  view.vector.block = v->block;
  view.vector.owner = 0;
  return view;
}

gsl_vector_const_view gsl_vector_const_subvector(const gsl_vector *v, size_t offset, size_t n) {
  SHIM_REQUIRE(offset + n <= v->size, "subvector out of range");
  _gsl_vector_const_view view;
  view.vector.size = n;
  view.vector.stride = v->stride;
  view.vector.data = v->data + offset * v->stride;
  view.vector.block = v->block;
  view.vector.owner = 0;
  return view;
}

gsl_vector_view gsl_vector_view_array(double *base, size_t n) {
  gsl_vector_view view;
  view.vector.size = n;
  view.vector.stride = 1;
  view.vector.data = base;
  view.vector.block = NULL;
  view.vector.owner = 0;
  return view;
}

gsl_vector_const_view gsl_vector_const_view_array(const double *base, size_t n) {
  _gsl_vector_const_view view;
  view.vector.size = n;
  view.vector.stride = 1;
  view.vector.data = (double *)base;
  view.vector.block = NULL;
  view.vector.owner = 0;
  return view;
}

int gsl_vector_fwrite(FILE *stream, const gsl_vector *v) {
  if (v->stride == 1) {
    size_t w = fwrite(v->data, sizeof(double), v->size, stream);
    return w == v->size ? GSL_SUCCESS : GSL_EINVAL;
  }
  for (size_t i = 0; i < v->size; ++i)
    if (fwrite(v->data + i * v->stride, sizeof(double), 1, stream) != 1) return GSL_EINVAL;
  return GSL_SUCCESS;
}

int gsl_vector_fread(FILE *stream, gsl_vector *v) {
  if (v->stride == 1) {
    size_t r = fread(v->data, sizeof(double), v->size, stream);
    return r == v->size ? GSL_SUCCESS : GSL_EINVAL;
  }
  for (size_t i = 0; i < v->size; ++i)
    if (fread(v->data + i * v->stride, sizeof(double), 1, stream) != 1) return GSL_EINVAL;
  return GSL_SUCCESS;
}

/* -------------------------------------------------------------- matrices */

static gsl_matrix *matrix_make(size_t n1, size_t n2, int zero) {
  gsl_matrix *m = (gsl_matrix *)malloc(sizeof(gsl_matrix));
  SHIM_REQUIRE(m != NULL, "matrix struct allocation failed");
  m->block = block_alloc(n1 * n2, zero);
  m->data = m->block->data;
  m->size1 = n1;
  m->size2 = n2;
  m->tda = n2;
  m->owner = 1;
  return m;
}

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2) { return matrix_make(n1, n2, 0); }
gsl_matrix *gsl_matrix_calloc(size_t n1, size_t n2) { return matrix_make(n1, n2, 1); }

void gsl_matrix_free(gsl_matrix *m) {
  if (!m) return;
  if (m->owner) block_free(m->block);
  free(m);
}

double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j) {
  SHIM_REQUIRE(i < m->size1 && j < m->size2, "matrix index out of range");
  return m->data[i * m->tda + j];
}

void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x) {
  SHIM_REQUIRE(i < m->size1 && j < m->size2, "matrix index out of range");
  m->data[i * m->tda + j] = x;
}

void gsl_matrix_set_zero(gsl_matrix *m) {
  for (size_t i = 0; i < m->size1; ++i)
    for (size_t j = 0; j < m->size2; ++j) m->data[i * m->tda + j] = 0.0;
}

int gsl_matrix_memcpy(gsl_matrix *dest, const gsl_matrix *src) {
  SHIM_REQUIRE(dest->size1 == src->size1 && dest->size2 == src->size2,
               "matrix shapes differ in memcpy");
  for (size_t i = 0; i < src->size1; ++i)
    for (size_t j = 0; j < src->size2; ++j)
      dest->data[i * dest->tda + j] = src->data[i * src->tda + j];
  return GSL_SUCCESS;
}

gsl_vector_view gsl_matrix_row(gsl_matrix *m, size_t i) {
  SHIM_REQUIRE(i < m->size1, "matrix row out of range");
  gsl_vector_view view;
  view.vector.size = m->size2;
  view.vector.stride = 1;
  view.vector.data = m->data + i * m->tda;
  view.vector.block = m->block;
  view.vector.owner = 0;
  return view;
}

gsl_vector_view gsl_matrix_column(gsl_matrix *m, size_t j) {
  SHIM_REQUIRE(j < m->size2, "matrix column out of range");
  gsl_vector_view view;
  view.vector.size = m->size1;
  view.vector.stride = m->tda;
  view.vector.data = m->data + j;
  view.vector.block = m->block;
  view.vector.owner = 0;
  return view;
}

gsl_vector_const_view gsl_matrix_const_row(const gsl_matrix *m, size_t i) {
  SHIM_REQUIRE(i < m->size1, "matrix row out of range");
  _gsl_vector_const_view view;
  view.vector.size = m->size2;
  view.vector.stride = 1;
  view.vector.data = m->data + i * m->tda;
  view.vector.block = m->block;
  view.vector.owner = 0;
  return view;
}

gsl_matrix_view gsl_matrix_view_vector(gsl_vector *v, size_t n1, size_t n2) {
  SHIM_REQUIRE(v->stride == 1 && n1 * n2 <= v->size, "matrix view of vector out of range");
  gsl_matrix_view view;
  view.matrix.size1 = n1;
  view.matrix.size2 = n2;
  view.matrix.tda = n2;
  view.matrix.data = v->data;
  view.matrix.block = v->block;
  view.matrix.owner = 0;
  return view;
}

gsl_matrix_const_view gsl_matrix_const_view_vector(const gsl_vector *v, size_t n1, size_t n2) {
  SHIM_REQUIRE(v->stride == 1 && n1 * n2 <= v->size, "matrix view of vector out of range");
  _gsl_matrix_const_view view;
  view.matrix.size1 = n1;
  view.matrix.size2 = n2;
  view.matrix.tda = n2;
  view.matrix.data = v->data;
  view.matrix.block = v->block;
  view.matrix.owner = 0;
  return view;
}

int gsl_matrix_fwrite(FILE *stream, const gsl_matrix *m) {
  if (m->tda == m->size2) {
    size_t n = m->size1 * m->size2;
    return fwrite(m->data, sizeof(double), n, stream) == n ? GSL_SUCCESS : GSL_EINVAL;
  }
  for (size_t i = 0; i < m->size1; ++i)
    if (fwrite(m->data + i * m->tda, sizeof(double), m->size2, stream) != m->size2)
      return GSL_EINVAL;
  return GSL_SUCCESS;
}

int gsl_matrix_fread(FILE *stream, gsl_matrix *m) {
  if (m->tda == m->size2) {
    size_t n = m->size1 * m->size2;
    return fread(m->data, sizeof(double), n, stream) == n ? GSL_SUCCESS : GSL_EINVAL;
  }
  for (size_t i = 0; i < m->size1; ++i)
    if (fread(m->data + i * m->tda, sizeof(double), m->size2, stream) != m->size2)
      return GSL_EINVAL;
  return GSL_SUCCESS;
}

/* ------------------------------------------------------------------ BLAS */

int gsl_blas_ddot(const gsl_vector *x, const gsl_vector *y, double *result) {
  SHIM_REQUIRE(x->size == y->size, "vector lengths differ in ddot");
  double r = 0.0;
  for (size_t i = 0; i < x->size; ++i) r += x->data[i * x->stride] * y->data[i * y->stride];
  *result = r;
  return GSL_SUCCESS;
}

/* Euclidean norm by the scaled sum-of-squares recurrence of the netlib
 * reference BLAS DNRM2 (Hammarling): keep the running maximum |x_k| as `scale`
 * and the sum of (|x_k|/scale)^2 as `ssq`, so no square overflows. */
double gsl_blas_dnrm2(const gsl_vector *x) {
  const size_t n = x->size;
  if (n == 0) return 0.0;
  if (n == 1) return fabs(x->data[0]);
  double scale = 0.0, ssq = 1.0;
  for (size_t i = 0; i < n; ++i) {
    const double xi = x->data[i * x->stride];
    if (xi == 0.0) continue;
    const double a = fabs(xi);
    if (scale < a) {
      const double r = scale / a;
      ssq = 1.0 + ssq * r * r;
      scale = a;
    } else {
      const double r = a / scale;
      ssq += r * r;
    }
  }
  return scale * sqrt(ssq);
}

void gsl_blas_dscal(double alpha, gsl_vector *x) {
  for (size_t i = 0; i < x->size; ++i) x->data[i * x->stride] *= alpha;
}

/* ------------------------------------------------------------------ math */

double gsl_pow_2(const double x) { return x * x; }
double gsl_pow_3(const double x) { return x * x * x; }
double gsl_pow_4(const double x) {
  const double x2 = x * x;
  return x2 * x2;
}
double gsl_pow_5(const double x) {
  const double x2 = x * x;
  return x2 * x2 * x;
}
double gsl_pow_6(const double x) {
  const double x2 = x * x;
  return x2 * x2 * x2;
}
double gsl_pow_7(const double x) {
  const double x2 = x * x;
  const double x4 = x2 * x2;
  return x4 * x2 * x;
}
double gsl_hypot(const double x, const double y) { return hypot(x, y); }
double gsl_hypot3(const double x, const double y, const double z) {
  return sqrt(x * x + y * y + z * z);
}

/* ----------------------------------------------------------- permutations */

gsl_permutation *gsl_permutation_alloc(size_t n) {
  gsl_permutation *p = (gsl_permutation *)malloc(sizeof(gsl_permutation));
  SHIM_REQUIRE(p != NULL, "permutation allocation failed");
  p->data = (size_t *)malloc((n ? n : 1) * sizeof(size_t));
  SHIM_REQUIRE(p->data != NULL, "permutation data allocation failed");
  p->size = n;
  return p;
}

gsl_permutation *gsl_permutation_calloc(size_t n) {
  gsl_permutation *p = gsl_permutation_alloc(n);
  gsl_permutation_init(p);
  return p;
}

void gsl_permutation_init(gsl_permutation *p) {
  for (size_t i = 0; i < p->size; ++i) p->data[i] = i;
}

void gsl_permutation_free(gsl_permutation *p) {
  if (!p) return;
  free(p->data);
  free(p);
}

size_t gsl_permutation_get(const gsl_permutation *p, size_t i) {
  SHIM_REQUIRE(i < p->size, "permutation index out of range");
  return p->data[i];
}

/* ------------------------------------------------------------------- LU */

/* Gaussian elimination with partial pivoting (row interchanges), column by
 * column: the pivot of column j is the largest |a_ij| on or below the
 * diagonal; rows are swapped in place and the swap recorded in p. */
int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum) {
  SHIM_REQUIRE(A->size1 == A->size2, "LU of a non-square matrix");
  SHIM_REQUIRE(p->size == A->size1, "permutation length != matrix size");
  const size_t n = A->size1, t = A->tda;
  double *a = A->data;
  gsl_permutation_init(p);
  *signum = 1;
  for (size_t j = 0; j + 1 < n; ++j) {
    size_t piv = j;
    double best = fabs(a[j * t + j]);
    for (size_t i = j + 1; i < n; ++i) {
      const double v = fabs(a[i * t + j]);
      if (v > best) {
        best = v;
        piv = i;
      }
    }
    if (piv != j) {
      for (size_t k = 0; k < n; ++k) {
        const double tmp = a[j * t + k];
        a[j * t + k] = a[piv * t + k];
        a[piv * t + k] = tmp;
      }
      const size_t tp = p->data[j];
      p->data[j] = p->data[piv];
      p->data[piv] = tp;
      *signum = -*signum;
    }
    const double ajj = a[j * t + j];
    if (ajj != 0.0) {
      for (size_t i = j + 1; i < n; ++i) {
        const double lij = a[i * t + j] / ajj;
        a[i * t + j] = lij;
        for (size_t k = j + 1; k < n; ++k) a[i * t + k] -= lij * a[j * t + k];
      }
    }
  }
  return GSL_SUCCESS;
}

int gsl_linalg_LU_solve(const gsl_matrix *LU, const gsl_permutation *p, const gsl_vector *b,
                        gsl_vector *x) {
  SHIM_REQUIRE(LU->size1 == LU->size2, "LU of a non-square matrix");
  const size_t n = LU->size1, t = LU->tda;
  SHIM_REQUIRE(p->size == n && b->size == n && x->size == n, "LU solve size mismatch");
  const double *a = LU->data;
  double *y = (double *)malloc((n ? n : 1) * sizeof(double));
  SHIM_REQUIRE(y != NULL, "LU solve allocation failed");
  for (size_t i = 0; i < n; ++i) y[i] = b->data[p->data[i] * b->stride];
  for (size_t i = 0; i < n; ++i) /* L y = P b, unit diagonal */
    for (size_t k = 0; k < i; ++k) y[i] -= a[i * t + k] * y[k];
  for (size_t ii = n; ii-- > 0;) { /* U x = y */
    for (size_t k = ii + 1; k < n; ++k) y[ii] -= a[ii * t + k] * y[k];
    y[ii] /= a[ii * t + ii];
  }
  for (size_t i = 0; i < n; ++i) x->data[i * x->stride] = y[i];
  free(y);
  return GSL_SUCCESS;
}
