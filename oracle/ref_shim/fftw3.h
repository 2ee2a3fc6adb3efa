/* Minimal stand-in for FFTW3's fftw3.h.  The P-MILOS hot path only reaches FFTW
 * when the control file sets "Use FFT for convolutions" = 1; every workload of
 * this project uses direct convolution, so the shim declares the types and the
 * entry points and its implementations (ref_shim.c) abort if ever called.
 * Like the real header, fftw_complex is the C99 complex type when <complex.h>
 * was included first (the reference always includes it first). */
#ifndef PM_SHIM_FFTW3_H
#define PM_SHIM_FFTW3_H
#include <stddef.h>
#if defined(_Complex_I) && defined(complex) && defined(I)
typedef double _Complex fftw_complex;
#else
typedef double fftw_complex[2];
#endif
typedef struct pm_shim_fftw_plan_s *fftw_plan;
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
void fftw_execute(const fftw_plan p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
#endif
