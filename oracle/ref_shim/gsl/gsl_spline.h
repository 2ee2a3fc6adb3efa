/* Minimal stand-in for GSL's interpolation API (gsl_interp.h / gsl_spline.h).
 * Only linear interpolation is implemented (interpolationLinearPSF uses it);
 * the cubic-spline entry points exist so that milosUtils.c links, and abort. */
#ifndef PM_SHIM_GSL_SPLINE_H
#define PM_SHIM_GSL_SPLINE_H
#include <stddef.h>
#include "gsl_math.h"
typedef struct { const char *name; int kind; } gsl_interp_type;
extern const gsl_interp_type *gsl_interp_linear;
extern const gsl_interp_type *gsl_interp_cspline;
typedef struct { size_t cache; } gsl_interp_accel;
typedef struct { const gsl_interp_type *type; size_t size; double xmin, xmax; } gsl_interp;
typedef struct { gsl_interp *interp; double *x; double *y; size_t size; } gsl_spline;
gsl_interp *gsl_interp_alloc(const gsl_interp_type *T, size_t n);
int gsl_interp_init(gsl_interp *interp, const double xa[], const double ya[], size_t size);
double gsl_interp_eval(const gsl_interp *interp, const double xa[], const double ya[], double x, gsl_interp_accel *a);
void gsl_interp_free(gsl_interp *interp);
gsl_interp_accel *gsl_interp_accel_alloc(void);
void gsl_interp_accel_free(gsl_interp_accel *a);
gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t size);
int gsl_spline_init(gsl_spline *spline, const double xa[], const double ya[], size_t size);
double gsl_spline_eval(const gsl_spline *spline, double x, gsl_interp_accel *a);
void gsl_spline_free(gsl_spline *spline);
#endif
