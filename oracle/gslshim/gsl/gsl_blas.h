/* Test infrastructure: level-1 BLAS subset of the GSL API (see gsl_shim_core.h). */
#ifndef PAWAN_ORACLE_GSL_BLAS_H
#define PAWAN_ORACLE_GSL_BLAS_H

#include "gsl_shim_core.h"
#include "gsl_vector.h"

#ifdef __cplusplus
extern "C" {
#endif

int gsl_blas_ddot(const gsl_vector *x, const gsl_vector *y, double *result);
double gsl_blas_dnrm2(const gsl_vector *x);
void gsl_blas_dscal(double alpha, gsl_vector *x);

#ifdef __cplusplus
}
#endif

#endif
