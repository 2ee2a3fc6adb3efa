/*
 * pm_oracle.h -- CPU restatement of P-MILOS's per-pixel Milne-Eddington inversion
 * (lm_mils and its callees).  TEST INFRASTRUCTURE ONLY: this is the checker that
 * the CUDA path is compared with.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it; the product never does.
 *
 * Built twice (oracle/Makefile): libpmoracle_f32.so with real = float and
 * libpmoracle_f64.so with real = double, mirroring the reference's REAL switch
 * (defines.h:8-36).  Model parameters, the wavelength grid, PSF taps and the
 * damped solve are double in both, as PRECISION is in the reference
 * (defines.h:59).
 *
 * Parity is pinned two ways (tests/test_oracle_*.py): against the reference's
 * own golden vector test/synthesis_results.per, and against the reference's
 * own C sources compiled unmodified into oracle/_ref/ (bit-for-bit when both are
 * built with the same flags), through fixtures committed under tests/golden/.
 */
#ifndef PM_ORACLE_H
#define PM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pmo_ctx pmo_ctx;

/* Per-pixel statistics that the reference computes but does not return. */
typedef struct {
  int iterations;   /* same value as lm_mils' *iter */
  int accepted;     /* LM steps that lowered chi^2 (each one re-ran me_der) */
  int status;       /* how lm_mils' loop ended: 0 the toplim test (or chi^2 < 1e-4),
                       1 the lambda bound, 2 the iteration cap; -1 nfree == 0
                       (lm_mils returns -1) -- the codes of pmilos.h's PM_PIX_* */
} pmo_stats;

int pmo_sizeof_real(void);

/* cuantic_dat[7] = {1, SLOI, LLOI, JLOI, SUPI, LUPI, JUPI} as readFileCuanticLines
 * (readConfig.c:24-129) produces it; psf = NULL for no instrumental profile,
 * else nlambda taps with the centre at nlambda/2. */
pmo_ctx *pmo_create(int nlambda, const double *lambda, double lambda0, const double *cuantic_dat,
                    const double *psf, int nterms);
void pmo_destroy(pmo_ctx *c);

/* Zeeman pattern (create_cuantic): N_PI, N_SIG, GL, GU, GEFF, FO, NUB, NUP, NUR, WEB, WEP, WER. */
int pmo_cuantic(const pmo_ctx *c, double *out, int cap);

/* mil_sinrf (+ me_der when d_spectra_out != NULL) at one model, as the reference's
 * synthesis mode runs them (milos.c:601-602). */
int pmo_synth(pmo_ctx *c, const double *model, const double *slight, double mu, const int *fix,
              double *spectra_out, double *d_spectra_out);

/* estimacionesClasicas(..., forInitialUse = 1) on one pixel. */
void pmo_classical(const pmo_ctx *c, const float *spectro, double *model_inout);
void pmo_classical_only(const pmo_ctx *c, const float *spectro, double *model_inout);

/* The per-pixel body of milos.c:958-1009: guess copy, optional classical estimates
 * with the NaN fixes, then lm_mils.  Returns lm_mils' return value (1 or -1). */
int pmo_invert_pixel(pmo_ctx *c, const float *spectro, const double *guess, const double *slight,
                     int use_classical, int miter, const double *w, double noise, double ilambda,
                     int logclambda, double toplim, double mu, const int *fix, double *model_out,
                     float *chisq, int *iters, double *spectra_out, pmo_stats *stats);

/* The same over npix pixels ([npix][4][nlambda] float32). slight: NULL, one
 * [4][nlambda] profile, or a [npix][4][nlambda] cube (slight_per_pixel = 1). */
int pmo_invert_batch(pmo_ctx *c, int npix, const float *spectro, const double *guess, const double *slight,
                     int slight_per_pixel, int use_classical, int miter, const double *w, double noise,
                     double ilambda, int logclambda, double toplim, double mu, const int *fix,
                     double *models_out, float *chisq_out, int *iters_out, float *spectra_out,
                     int *accepted_out, int *status_out);

/* Unit-level pieces. */
int pmo_fvoigt(double damp, const double *v, int n, double *h, double *f);
int pmo_conv(const pmo_ctx *c, double *x, int mode, double ic);
/* mil_svd semantics: eigen-decompose covar (K x K, destroyed), pseudo-inverse with
 * |w| <= 1e-12 eigenvalues dropped, delta = V diag(1/w) V^T beta. */
int pmo_svd_solve(int K, double *covar, const double *beta, double *delta);

#ifdef __cplusplus
}
#endif
#endif
