/* Empty stand-in for GSL gsl_blas.h: lib.c includes it but calls nothing from it. */
#ifndef PM_SHIM_GSL_BLAS_H
#define PM_SHIM_GSL_BLAS_H
#include "gsl_matrix.h"
#endif
