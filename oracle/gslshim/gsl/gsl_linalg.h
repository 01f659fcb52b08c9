/* Test infrastructure: the LU subset of the GSL linear-algebra API (see
 * gsl_shim_core.h), used by the reference's resolve path. */
#ifndef PAWAN_ORACLE_GSL_LINALG_H
#define PAWAN_ORACLE_GSL_LINALG_H

#include "gsl_matrix.h"
#include "gsl_permutation.h"
#include "gsl_vector.h"

#ifdef __cplusplus
extern "C" {
#endif

/* P A = L U with partial pivoting, in place: L (unit diagonal) below the
 * diagonal, U on and above it; signum = sign of the permutation. */
int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum);
/* Solves A x = b from the factors of gsl_linalg_LU_decomp. */
int gsl_linalg_LU_solve(const gsl_matrix *LU, const gsl_permutation *p, const gsl_vector *b,
                        gsl_vector *x);

#ifdef __cplusplus
}
#endif

#endif
