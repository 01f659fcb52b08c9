/* Test infrastructure: matrix subset of the GSL API (see gsl_shim_core.h). */
#ifndef PAWAN_ORACLE_GSL_MATRIX_H
#define PAWAN_ORACLE_GSL_MATRIX_H

#include "gsl_shim_core.h"
#include "gsl_vector.h"

#ifdef __cplusplus
extern "C" {
#endif

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
gsl_matrix *gsl_matrix_calloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);

double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j);
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x);
void gsl_matrix_set_zero(gsl_matrix *m);
int gsl_matrix_memcpy(gsl_matrix *dest, const gsl_matrix *src);

gsl_vector_view gsl_matrix_row(gsl_matrix *m, size_t i);
gsl_vector_view gsl_matrix_column(gsl_matrix *m, size_t j);
gsl_vector_const_view gsl_matrix_const_row(const gsl_matrix *m, size_t i);
gsl_matrix_view gsl_matrix_view_vector(gsl_vector *v, size_t n1, size_t n2);
gsl_matrix_const_view gsl_matrix_const_view_vector(const gsl_vector *v, size_t n1, size_t n2);

int gsl_matrix_fwrite(FILE *stream, const gsl_matrix *m);
int gsl_matrix_fread(FILE *stream, gsl_matrix *m);

#ifdef __cplusplus
}
#endif

#endif
