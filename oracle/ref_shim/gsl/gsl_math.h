/* Minimal stand-in for GSL's gsl_math.h (test infrastructure for the oracle). */
#ifndef PM_SHIM_GSL_MATH_H
#define PM_SHIM_GSL_MATH_H
#include <math.h>
#define GSL_NAN (NAN)
int gsl_isnan(const double x);
#endif
