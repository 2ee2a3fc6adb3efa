/* Minimal stand-in for GSL's gsl_eigen.h: the real symmetric eigen-solver with
 * eigenvectors (gsl_eigen_symmv).  The implementation in ref_shim.c is a cyclic
 * Jacobi method written from the textbook mathematics; like GSL it reads the
 * diagonal and lower triangle of A only and destroys them, returns unordered
 * eigenvalues in eval and the matching orthonormal eigenvectors as the columns
 * of evec. */
#ifndef PM_SHIM_GSL_EIGEN_H
#define PM_SHIM_GSL_EIGEN_H
#include "gsl_vector.h"
#include "gsl_matrix.h"
typedef struct {
  size_t size;
  double *work;
} gsl_eigen_symmv_workspace;
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(const size_t n);
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w);
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w);
#endif
