/* Minimal stand-in for GSL's gsl_matrix.h: a dense row-major double matrix. */
#ifndef PM_SHIM_GSL_MATRIX_H
#define PM_SHIM_GSL_MATRIX_H
#include <stddef.h>
#include "gsl_vector.h"
typedef struct {
  size_t size1;
  size_t size2;
  size_t tda;
  double *data;
  void *block;
  int owner;
} gsl_matrix;
typedef struct {
  gsl_matrix matrix;
} gsl_matrix_view;
gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2);
double *gsl_matrix_ptr(gsl_matrix *m, size_t i, size_t j);
#endif
