/*
 * ref_shim.c -- project-written implementations of the few GSL and FFTW entry
 * points that the P-MILOS hot-path sources call (TEST INFRASTRUCTURE ONLY).
 *
 * The reference links GSL (gsl_eigen_symmv, gsl_interp_linear) and FFTW3; neither
 * library exists in this environment, and neither is vendored by the reference,
 * so the oracle build links these shims instead:
 *
 *  - gsl_eigen_symmv: cyclic Jacobi eigen-decomposition of a real symmetric
 *    matrix (pm_jacobi.h, written from the textbook method).  Same contract as GSL: reads the diagonal and lower triangle of A,
 *    returns unordered eigenvalues and orthonormal eigenvectors as the columns of
 *    evec (row-major, v[i*n+j] = component i of eigenvector j).  The caller
 *    (mil_svd, milosUtils.c:237-271) only forms V diag(1/w) V^T beta, which does
 *    not depend on eigenvalue order or eigenvector signs.
 *  - gsl_interp_linear: piecewise-linear interpolation; out-of-range x returns NaN
 *    (interpolationLinearPSF, milosUtils.c:684-738, maps NaN to 0).
 *  - FFTW3 and cubic splines: reached only when "Use FFT" = 1 or by the unused
 *    interpolationSplinePSF; they abort so that an accidental call is loud.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>
#include "fftw3.h"
#include "gsl/gsl_math.h"
#include "gsl/gsl_vector.h"
#include "gsl/gsl_matrix.h"
#include "gsl/gsl_eigen.h"
#include "gsl/gsl_spline.h"
#include "../pm_jacobi.h"

static void shim_unreachable(const char *what) {
  fprintf(stderr, "oracle shim: %s is not available in the oracle build\n", what);
  abort();
}

int gsl_isnan(const double x) { return isnan(x) ? 1 : 0; }

gsl_vector *gsl_vector_alloc(size_t n) {
  gsl_vector *v = (gsl_vector *)calloc(1, sizeof(gsl_vector));
  v->size = n;
  v->stride = 1;
  v->data = (double *)calloc(n ? n : 1, sizeof(double));
  v->owner = 1;
  return v;
}
void gsl_vector_free(gsl_vector *v) {
  if (!v) return;
  if (v->owner) free(v->data);
  free(v);
}
double *gsl_vector_ptr(gsl_vector *v, size_t i) { return v->data + i * v->stride; }

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2) {
  gsl_matrix *m = (gsl_matrix *)calloc(1, sizeof(gsl_matrix));
  m->size1 = n1;
  m->size2 = n2;
  m->tda = n2;
  m->data = (double *)calloc(n1 * n2 ? n1 * n2 : 1, sizeof(double));
  m->owner = 1;
  return m;
}
void gsl_matrix_free(gsl_matrix *m) {
  if (!m) return;
  if (m->owner) free(m->data);
  free(m);
}
gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2) {
  gsl_matrix_view view;
  memset(&view, 0, sizeof(view));
  view.matrix.size1 = n1;
  view.matrix.size2 = n2;
  view.matrix.tda = n2;
  view.matrix.data = base;
  view.matrix.owner = 0;
  return view;
}
double *gsl_matrix_ptr(gsl_matrix *m, size_t i, size_t j) { return m->data + i * m->tda + j; }

gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(const size_t n) {
  gsl_eigen_symmv_workspace *w = (gsl_eigen_symmv_workspace *)calloc(1, sizeof(*w));
  w->size = n;
  w->work = (double *)calloc(n * n ? n * n : 1, sizeof(double));
  return w;
}
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w) {
  if (!w) return;
  free(w->work);
  free(w);
}

/* gsl_eigen_symmv on top of the shared Jacobi routine: copy the diagonal and
 * lower triangle into a full symmetric work matrix, decompose, then clear the
 * lower triangle of A as GSL documents it destroys it. */
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *ws) {
  const size_t n = A->size1;
  double *a = ws->work;
  double wv[64], vv[64 * 64];
  size_t i, j;
  if (n > 64) shim_unreachable("gsl_eigen_symmv with n > 64");
  for (i = 0; i < n; i++)
    for (j = 0; j <= i; j++) {
      double x = A->data[i * A->tda + j];
      a[i * n + j] = x;
      a[j * n + i] = x;
    }
  pm_jacobi_eigen(a, n, wv, vv);
  for (i = 0; i < n; i++) {
    eval->data[i * eval->stride] = wv[i];
    for (j = 0; j < n; j++) evec->data[i * evec->tda + j] = vv[i * n + j];
  }
  for (i = 0; i < n; i++)
    for (j = 0; j <= i; j++) A->data[i * A->tda + j] = 0.0;
  return 0;
}

static const gsl_interp_type shim_linear = {"linear", 1};
static const gsl_interp_type shim_cspline = {"cspline", 2};
const gsl_interp_type *gsl_interp_linear = &shim_linear;
const gsl_interp_type *gsl_interp_cspline = &shim_cspline;

gsl_interp *gsl_interp_alloc(const gsl_interp_type *T, size_t n) {
  gsl_interp *it;
  if (T != gsl_interp_linear) shim_unreachable("non-linear gsl_interp");
  it = (gsl_interp *)calloc(1, sizeof(gsl_interp));
  it->type = T;
  it->size = n;
  return it;
}
int gsl_interp_init(gsl_interp *interp, const double xa[], const double ya[], size_t size) {
  (void)ya;
  interp->xmin = xa[0];
  interp->xmax = xa[size - 1];
  interp->size = size;
  return 0;
}
/* Linear interpolation on a strictly increasing abscissa: locate i with
 * xa[i] <= x < xa[i+1] by bisection (the last interval is closed on the right),
 * then y = y_i + (x - x_i)/(x_{i+1} - x_i) * (y_{i+1} - y_i). */
double gsl_interp_eval(const gsl_interp *interp, const double xa[], const double ya[], double x, gsl_interp_accel *acc) {
  size_t lo = 0, hi = interp->size - 1;
  double dx;
  (void)acc;
  if (!(x >= interp->xmin && x <= interp->xmax)) return GSL_NAN;
  while (hi > lo + 1) {
    size_t mid = (lo + hi) / 2;
    if (xa[mid] > x)
      hi = mid;
    else
      lo = mid;
  }
  dx = xa[lo + 1] - xa[lo];
  if (!(dx > 0.0)) return 0.0;
  return ya[lo] + (x - xa[lo]) / dx * (ya[lo + 1] - ya[lo]);
}
void gsl_interp_free(gsl_interp *interp) { free(interp); }
gsl_interp_accel *gsl_interp_accel_alloc(void) { return (gsl_interp_accel *)calloc(1, sizeof(gsl_interp_accel)); }
void gsl_interp_accel_free(gsl_interp_accel *a) { free(a); }
gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t size) {
  (void)T; (void)size;
  shim_unreachable("gsl_spline_alloc");
  return NULL;
}
int gsl_spline_init(gsl_spline *spline, const double xa[], const double ya[], size_t size) {
  (void)spline; (void)xa; (void)ya; (void)size;
  shim_unreachable("gsl_spline_init");
  return 0;
}
double gsl_spline_eval(const gsl_spline *spline, double x, gsl_interp_accel *a) {
  (void)spline; (void)x; (void)a;
  shim_unreachable("gsl_spline_eval");
  return 0.0;
}
void gsl_spline_free(gsl_spline *spline) { (void)spline; }

void fftw_execute(const fftw_plan p) { (void)p; shim_unreachable("fftw_execute"); }
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
  (void)n; (void)in; (void)out; (void)sign; (void)flags;
  shim_unreachable("fftw_plan_dft_1d");
  return NULL;
}
void fftw_destroy_plan(fftw_plan p) { (void)p; }
void *fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void *p) { free(p); }
