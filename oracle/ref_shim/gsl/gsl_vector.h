/* Minimal stand-in for GSL's gsl_vector.h: a dense double vector with unit stride. */
#ifndef PM_SHIM_GSL_VECTOR_H
#define PM_SHIM_GSL_VECTOR_H
#include <stddef.h>
typedef struct {
  size_t size;
  size_t stride;
  double *data;
  void *block;
  int owner;
} gsl_vector;
gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double *gsl_vector_ptr(gsl_vector *v, size_t i);
#endif
