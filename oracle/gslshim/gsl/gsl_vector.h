/* Test infrastructure: vector subset of the GSL API (see gsl_shim_core.h). */
#ifndef PAWAN_ORACLE_GSL_VECTOR_H
#define PAWAN_ORACLE_GSL_VECTOR_H

#include "gsl_shim_core.h"

#ifdef __cplusplus
extern "C" {
#endif

gsl_vector *gsl_vector_alloc(size_t n);
gsl_vector *gsl_vector_calloc(size_t n);
void gsl_vector_free(gsl_vector *v);

double gsl_vector_get(const gsl_vector *v, size_t i);
void gsl_vector_set(gsl_vector *v, size_t i, double x);
double *gsl_vector_ptr(gsl_vector *v, size_t i);
void gsl_vector_set_zero(gsl_vector *v);
void gsl_vector_set_all(gsl_vector *v, double x);

int gsl_vector_memcpy(gsl_vector *dest, const gsl_vector *src);
int gsl_vector_add(gsl_vector *a, const gsl_vector *b);
int gsl_vector_sub(gsl_vector *a, const gsl_vector *b);
int gsl_vector_mul(gsl_vector *a, const gsl_vector *b);
int gsl_vector_scale(gsl_vector *a, double x);
int gsl_vector_add_constant(gsl_vector *a, double x);

gsl_vector_view gsl_vector_subvector(gsl_vector *v, size_t offset, size_t n);
gsl_vector_const_view gsl_vector_const_subvector(const gsl_vector *v, size_t offset, size_t n);
gsl_vector_view gsl_vector_view_array(double *base, size_t n);
gsl_vector_const_view gsl_vector_const_view_array(const double *base, size_t n);

int gsl_vector_fwrite(FILE *stream, const gsl_vector *v);
int gsl_vector_fread(FILE *stream, gsl_vector *v);

#ifdef __cplusplus
}
#endif

#endif
