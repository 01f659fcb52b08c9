/* Test infrastructure: permutation subset of the GSL API (see gsl_shim_core.h). */
#ifndef PAWAN_ORACLE_GSL_PERMUTATION_H
#define PAWAN_ORACLE_GSL_PERMUTATION_H

#include "gsl_shim_core.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  size_t size;
  size_t *data;
} gsl_permutation;

gsl_permutation *gsl_permutation_alloc(size_t n);
gsl_permutation *gsl_permutation_calloc(size_t n);
void gsl_permutation_init(gsl_permutation *p);
void gsl_permutation_free(gsl_permutation *p);
size_t gsl_permutation_get(const gsl_permutation *p, size_t i);

#ifdef __cplusplus
}
#endif

#endif
