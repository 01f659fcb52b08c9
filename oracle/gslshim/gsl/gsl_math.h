/* Test infrastructure: math constants and small power helpers of the GSL API
 * (see gsl_shim_core.h).  The powers are out-of-line calls, as in a default GSL
 * build without HAVE_INLINE. */
#ifndef PAWAN_ORACLE_GSL_MATH_H
#define PAWAN_ORACLE_GSL_MATH_H

#include <math.h>
#include "gsl_shim_core.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846264338328
#endif
#ifndef M_1_PI
#define M_1_PI 0.31830988618379067153776752675
#endif

#ifdef __cplusplus
extern "C" {
#endif

double gsl_pow_2(const double x);
double gsl_pow_3(const double x);
double gsl_pow_4(const double x);
double gsl_pow_5(const double x);
double gsl_pow_6(const double x);
double gsl_pow_7(const double x);
double gsl_hypot(const double x, const double y);
double gsl_hypot3(const double x, const double y, const double z);

#ifdef __cplusplus
}
#endif

#endif
