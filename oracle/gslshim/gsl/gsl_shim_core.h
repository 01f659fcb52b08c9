/* Test infrastructure: a minimal, project-written stand-in for the subset of the
 * GNU Scientific Library API that pawan's hot path uses.  GSL itself is not
 * installed in this image, so the reference's own sources are compiled against
 * these headers to serve as the parity oracle.  Only the public API semantics
 * are followed (struct member names, argument order, return codes); nothing
 * here is GSL source.
 *
 * Behavioural choices that matter for parity and for the CPU baseline:
 *   - gsl_vector_get/set and gsl_matrix_get/set are out-of-line and
 *     range-checked, as they are in a default (non-HAVE_INLINE) GSL build;
 *   - *_calloc makes three allocations (container, block, data), as GSL does;
 *   - gsl_blas_dnrm2 uses the scaled sum-of-squares recurrence of the netlib
 *     reference BLAS DNRM2, which is what GSL's CBLAS implements;
 *   - any size mismatch or out-of-range index aborts, like GSL's default
 *     error handler.
 */
#ifndef PAWAN_ORACLE_GSL_SHIM_CORE_H
#define PAWAN_ORACLE_GSL_SHIM_CORE_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { GSL_SUCCESS = 0, GSL_EBADLEN = 19, GSL_EINVAL = 4 };

typedef struct {
  size_t size;
  double *data;
} gsl_block;

typedef struct {
  size_t size;
  size_t stride;
  double *data;
  gsl_block *block;
  int owner;
} gsl_vector;

typedef struct {
  gsl_vector vector;
} _gsl_vector_view;
typedef _gsl_vector_view gsl_vector_view;

typedef struct {
  gsl_vector vector;
} _gsl_vector_const_view;
typedef const _gsl_vector_const_view gsl_vector_const_view;

typedef struct {
  size_t size1;
  size_t size2;
  size_t tda;
  double *data;
  gsl_block *block;
  int owner;
} gsl_matrix;

typedef struct {
  gsl_matrix matrix;
} _gsl_matrix_view;
typedef _gsl_matrix_view gsl_matrix_view;

typedef struct {
  gsl_matrix matrix;
} _gsl_matrix_const_view;
typedef const _gsl_matrix_const_view gsl_matrix_const_view;

/* error path shared by every checked call: print and abort */
void gslshim_fail(const char *what, const char *file, int line);

#ifdef __cplusplus
}
#endif

#endif
