/* Empty stand-in for GSL gsl_cblas.h: lib.c includes it but calls nothing from it. */
#ifndef PM_SHIM_GSL_CBLAS_H
#define PM_SHIM_GSL_CBLAS_H
#include "gsl_matrix.h"
#endif
