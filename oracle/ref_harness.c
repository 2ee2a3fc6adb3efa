/*
 * ref_harness.c -- driver for the REFERENCE's own hot-path C code (TEST
 * INFRASTRUCTURE ONLY; built into oracle/_ref/ by oracle/Makefile, never shipped).
 *
 * The P-MILOS hot path (mil_sinrf.c, me_der.c, fvoigt.c, convolution.c, lib.c,
 * milosUtils.c, create_cuantic.c, calculosCompartidos.c, fgauss.c) is compiled
 * unmodified from the reference tree.  Those files expect their process-wide
 * state (NTERMS, cuantic, G, ~60 scratch arrays, the GSL workspace, ...) to be
 * defined by the driver program; this file plays the role of that driver the way
 * src/milos.c does (milos.c:39-100 declare the same globals -- the names and
 * types must match for the link to succeed) and exposes a small C API that the
 * Python test suite and the CPU baseline call through ctypes:
 *
 *   pmref_setup        line data + wavelength grid + PSF taps + NTERMS
 *                      (milos.c:143-230 globals; create_cuantic, AllocateMemoryDerivedSynthesis)
 *   pmref_synth        mil_sinrf + me_der at one model (synthesis mode, milos.c:601-602)
 *   pmref_classical    estimacionesClasicas (milosUtils.c:287-452)
 *   pmref_classical_only the same with forInitialUse = 0 (milos.c:486-501)
 *   pmref_invert_pixel the per-pixel body of milos.c:958-1009: guess copy,
 *                      classical estimates, NaN fixes, lm_mils
 *   pmref_invert_batch the same over a contiguous slab of pixels (CPU baseline)
 *   pmref_* helpers    fvoigt, the direct convolutions, covarm2, fchisqr, mil_svd,
 *                      fgauss_WL, interpolationLinearPSF for unit-level pinning.
 *
 * REAL is float by default and double with -DUSE_DOUBLE_PRECISION=double, exactly
 * like the reference makefile (makefile:22-26); this API converts REAL arrays to
 * and from double so one ctypes binding serves both builds.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>
#include "defines.h"
#include <fftw3.h>
#include <gsl/gsl_eigen.h>
#include "milosUtils.h"
#include "lib.h"
#include "convolution.h"

/* ---- process-wide state the reference sources reference as extern ---- */
int NTERMS = 11;
Cuantic *cuantic = NULL;
PRECISION **PUNTEROS_CALCULOS_COMPARTIDOS;
int POSW_PUNTERO_CALCULOS_COMPARTIDOS;
int POSR_PUNTERO_CALCULOS_COMPARTIDOS;
REAL *dtaux, *etai_gp3, *ext1, *ext2, *ext3, *ext4;
REAL *gp1, *gp2, *dt, *dti, *gp3, *gp4, *gp5, *gp6, *etai_2;
REAL *gp4_gp2_rhoq, *gp5_gp2_rhou, *gp6_gp2_rhov;
REAL *dgp1, *dgp2, *dgp3, *dgp4, *dgp5, *dgp6, *d_dt;
REAL *d_ei, *d_eq, *d_eu, *d_ev, *d_rq, *d_ru, *d_rv;
REAL *dfi, *dshi;
REAL CC, CC_2, sin_gm, azi_2, sinis, cosis, cosis_2, cosi, sina, cosa, sinda, cosda, sindi, cosdi, sinis_cosa, sinis_sina;
REAL *fi_p, *fi_b, *fi_r, *shi_p, *shi_b, *shi_r;
REAL *etain, *etaqn, *etaun, *etavn, *rhoqn, *rhoun, *rhovn;
REAL *etai, *etaq, *etau, *etav, *rhoq, *rhou, *rhov;
REAL *parcial1, *parcial2, *parcial3;
REAL *nubB, *nupB, *nurB;
REAL **uuGlobalInicial;
REAL **HGlobalInicial;
REAL **FGlobalInicial;
PRECISION *GMAC, *GMAC_DERIV;
PRECISION *dirConvPar;
REAL *resultConv;
PRECISION *G = NULL;
REAL *opa;
int FGlobal, HGlobal, uuGlobal;
REAL *d_spectra, *spectra, *spectra_mac, *spectra_slight;
fftw_complex *inSpectraFwPSF, *inSpectraBwPSF, *outSpectraFwPSF, *outSpectraBwPSF;
fftw_complex *inSpectraFwMAC, *inSpectraBwMAC, *outSpectraFwMAC, *outSpectraBwMAC;
fftw_plan planForwardPSF, planBackwardPSF;
fftw_plan planForwardMAC, planBackwardMAC;
fftw_complex *inFilterMAC, *inFilterMAC_DERIV, *outFilterMAC, *outFilterMAC_DERIV;
fftw_plan planFilterMAC, planFilterMAC_DERIV;
fftw_complex *fftw_G_PSF, *fftw_G_MAC_PSF, *fftw_G_MAC_DERIV_PSF;
fftw_complex *inPSF_MAC, *inMulMacPSF, *inPSF_MAC_DERIV, *inMulMacPSFDeriv, *outConvFilters, *outConvFiltersDeriv;
fftw_plan planForwardPSF_MAC, planForwardPSF_MAC_DERIV, planBackwardPSF_MAC, planBackwardPSF_MAC_DERIV;
int sizeG = 0;
PRECISION FWHM = 0;
ConfigControl configCrontrolFile;
_Complex double *z, *zden, *zdiv;
gsl_vector *eval;
gsl_matrix *evec;
gsl_eigen_symmv_workspace *workspace;

/* ---- harness-private state ---- */
static int h_nl = 0;
static PRECISION h_wlines[2];
static PRECISION *h_lambda = NULL;
static int h_filter = 0;
static REAL *h_vsigma = NULL;
static REAL *h_slight = NULL;
static int h_ready = 0;

static void model_from(Init_Model *m, const double *p) {
  m->eta0 = p[0]; m->B = p[1]; m->vlos = p[2]; m->dopp = p[3]; m->aa = p[4];
  m->gm = p[5]; m->az = p[6]; m->S0 = p[7]; m->S1 = p[8]; m->mac = p[9]; m->alfa = p[10];
}
static void model_to(double *p, const Init_Model *m) {
  p[0] = m->eta0; p[1] = m->B; p[2] = m->vlos; p[3] = m->dopp; p[4] = m->aa;
  p[5] = m->gm; p[6] = m->az; p[7] = m->S0; p[8] = m->S1; p[9] = m->mac; p[10] = m->alfa;
}

int pmref_sizeof_real(void) { return (int)sizeof(REAL); }

void pmref_teardown(void) {
  if (!h_ready) return;
  FreeMemoryDerivedSynthesis();
  if (cuantic) {
    free(cuantic[0].NUB); free(cuantic[0].NUP); free(cuantic[0].NUR);
    free(cuantic[0].WEB); free(cuantic[0].WEP); free(cuantic[0].WER);
    free(cuantic);
    cuantic = NULL;
  }
  gsl_vector_free(eval);
  gsl_matrix_free(evec);
  gsl_eigen_symmv_free(workspace);
  free(h_lambda); h_lambda = NULL;
  free(G); G = NULL;
  free(h_vsigma); h_vsigma = NULL;
  free(h_slight); h_slight = NULL;
  h_ready = 0;
}

/* cuantic_dat[7] = {nlines(=1), SLOI, LLOI, JLOI, SUPI, LUPI, JUPI}, i.e. what
 * readFileCuanticLines (readConfig.c:24-129) writes.  psf = NULL disables the
 * instrumental convolution.  Returns 0 on success. */
int pmref_setup(int nlambda, const double *lambda, double lambda0, const double *cuantic_dat,
                const double *psf, int nterms) {
  int i;
  pmref_teardown();
  if (nlambda <= 0 || nterms < 1 || nterms > 11) return -1;
  memset(&configCrontrolFile, 0, sizeof(configCrontrolFile));
  configCrontrolFile.useFFT = 0;
  NTERMS = nterms;
  CC = PI / 180.0;
  CC_2 = CC * 2;
  h_nl = nlambda;
  h_wlines[0] = 1;
  h_wlines[1] = lambda0;
  h_lambda = (PRECISION *)malloc(sizeof(PRECISION) * nlambda);
  for (i = 0; i < nlambda; i++) h_lambda[i] = lambda[i];
  {
    PRECISION dat[7];
    for (i = 0; i < 7; i++) dat[i] = cuantic_dat[i];
    cuantic = create_cuantic(dat, 0);
  }
  eval = gsl_vector_alloc(NTERMS);
  evec = gsl_matrix_alloc(NTERMS, NTERMS);
  workspace = gsl_eigen_symmv_alloc(NTERMS);
  if (psf) {
    G = (PRECISION *)malloc(sizeof(PRECISION) * nlambda);
    for (i = 0; i < nlambda; i++) G[i] = psf[i];
    sizeG = nlambda;
    h_filter = 1;
  } else {
    G = NULL;
    sizeG = 0;
    h_filter = 0;
  }
  AllocateMemoryDerivedSynthesis(nlambda);
  h_vsigma = (REAL *)calloc(nlambda * NPARMS, sizeof(REAL));
  h_slight = (REAL *)calloc(nlambda * NPARMS, sizeof(REAL));
  h_ready = 1;
  return 0;
}

/* Zeeman pattern computed by create_cuantic for the current line:
 * out[0..5] = N_PI, N_SIG, GL, GU, GEFF, FO; then NUB, NUP, NUR, WEB, WEP, WER. */
int pmref_cuantic(double *out, int cap) {
  int k = 0, i, ns, np;
  if (!h_ready) return -1;
  ns = (int)cuantic[0].N_SIG;
  np = (int)cuantic[0].N_PI;
  if (cap < 6 + 4 * ns + 2 * np) return -2;
  out[k++] = cuantic[0].N_PI; out[k++] = cuantic[0].N_SIG; out[k++] = cuantic[0].GL;
  out[k++] = cuantic[0].GU; out[k++] = cuantic[0].GEFF; out[k++] = cuantic[0].FO;
  for (i = 0; i < ns; i++) out[k++] = cuantic[0].NUB[i];
  for (i = 0; i < np; i++) out[k++] = cuantic[0].NUP[i];
  for (i = 0; i < ns; i++) out[k++] = cuantic[0].NUR[i];
  for (i = 0; i < ns; i++) out[k++] = cuantic[0].WEB[i];
  for (i = 0; i < np; i++) out[k++] = cuantic[0].WEP[i];
  for (i = 0; i < ns; i++) out[k++] = cuantic[0].WER[i];
  return k;
}

static REAL *stage_slight(const double *slight) {
  int i;
  if (!slight) return NULL;
  for (i = 0; i < h_nl * NPARMS; i++) h_slight[i] = (REAL)slight[i];
  return h_slight;
}

/* Synthesis at one model: mil_sinrf then me_der, as milos.c:601-602 does in
 * synthesis mode (no FijaACeroDerivadasNoNecesarias). */
int pmref_synth(const double *model, const double *slight, double mu, const int *fix,
                double *spectra_out, double *d_spectra_out) {
  Init_Model m;
  int i, fx[11];
  REAL *sl;
  if (!h_ready) return -1;
  model_from(&m, model);
  for (i = 0; i < 11; i++) fx[i] = fix ? fix[i] : 1;
  sl = stage_slight(slight);
  mil_sinrf(cuantic, &m, h_wlines, h_lambda, h_nl, spectra, (REAL)mu, sl, spectra_mac, spectra_slight, h_filter);
  if (spectra_out)
    for (i = 0; i < h_nl * NPARMS; i++) spectra_out[i] = spectra[i];
  if (d_spectra_out) {
    me_der(cuantic, &m, h_wlines, h_lambda, h_nl, d_spectra, spectra_mac, spectra_slight, (REAL)mu, sl, h_filter, fx);
    for (i = 0; i < h_nl * NPARMS * NTERMS; i++) d_spectra_out[i] = d_spectra[i];
  }
  return 0;
}

void pmref_classical(const float *spectro, double *model_inout) {
  Init_Model m;
  model_from(&m, model_inout);
  estimacionesClasicas(h_wlines[1], h_lambda, h_nl, (float *)spectro, &m, 1);
  model_to(model_inout, &m);
}

/* The per-pixel body of the classical-estimates-only mode, milos.c:486-501
 * (NumberOfCycles < 0): the initial model, then estimacionesClasicas with
 * forInitialUse = 0, nothing else. */
void pmref_classical_only(const float *spectro, double *model_inout) {
  Init_Model m;
  model_from(&m, model_inout);
  estimacionesClasicas(h_wlines[1], h_lambda, h_nl, (float *)spectro, &m, 0);
  model_to(model_inout, &m);
}

/* One pixel of milos.c:958-1009. */
int pmref_invert_pixel(const float *spectro, const double *guess, const double *slight, int use_classical,
                       int miter, const double *w, double noise, double ilambda, int logclambda,
                       double toplim, double mu, const int *fix, double *model_out, float *chisq,
                       int *iters, double *spectra_out) {
  Init_Model m;
  REAL weight[4];
  int i, it = -1, rc, fx[11], filt = h_filter;
  float chi = 0.0f;
  REAL *sl;
  if (!h_ready) return -100;
  for (i = 0; i < 4; i++) weight[i] = (REAL)w[i];
  for (i = 0; i < 11; i++) fx[i] = fix[i];
  model_from(&m, guess);
  if (use_classical) {
    estimacionesClasicas(h_wlines[1], h_lambda, h_nl, (float *)spectro, &m, 1);
    if (isnan(m.B)) m.B = 1;
    if (isnan(m.vlos)) m.vlos = 1e-3;
    if (isnan(m.gm)) m.gm = 1;
    if (isnan(m.az)) m.az = 1;
  }
  sl = stage_slight(slight);
  rc = lm_mils(cuantic, h_wlines, h_lambda, h_nl, (float *)spectro, h_nl, &m, spectra, &chi, sl, toplim, miter,
               weight, fx, h_vsigma, (REAL)noise, (REAL)ilambda, &filt, &it, (REAL)mu, logclambda);
  model_to(model_out, &m);
  if (chisq) *chisq = chi;
  if (iters) *iters = it;
  if (spectra_out)
    for (i = 0; i < h_nl * NPARMS; i++) spectra_out[i] = spectra[i];
  return rc;
}

/* A contiguous slab of pixels, [npix][4][nl] float32 in, models/chi2/iters out.
 * slight: NULL, one [4][nl] profile for all pixels, or a [npix][4][nl] cube
 * (slight_per_pixel = 1).  spectra_out (nullable) is [npix][4][nl] float32. */
int pmref_invert_batch(int npix, const float *spectro, const double *guess, const double *slight,
                       int slight_per_pixel, int use_classical, int miter, const double *w, double noise,
                       double ilambda, int logclambda, double toplim, double mu, const int *fix,
                       double *models_out, float *chisq_out, int *iters_out, float *spectra_out) {
  int p, i;
  double *sp = spectra_out ? (double *)malloc(sizeof(double) * h_nl * NPARMS) : NULL;
  for (p = 0; p < npix; p++) {
    const double *slp = slight ? (slight_per_pixel ? slight + (size_t)p * h_nl * NPARMS : slight) : NULL;
    pmref_invert_pixel(spectro + (size_t)p * h_nl * NPARMS, guess, slp, use_classical, miter, w, noise, ilambda,
                       logclambda, toplim, mu, fix, models_out + (size_t)p * 11, chisq_out + p, iters_out + p, sp);
    if (sp)
      for (i = 0; i < h_nl * NPARMS; i++) spectra_out[(size_t)p * h_nl * NPARMS + i] = (float)sp[i];
  }
  free(sp);
  return 0;
}

/* ---- unit-level entry points ---- */
int pmref_fvoigt(double damp, const double *v, int n, double *h, double *f) {
  REAL *vv = malloc(sizeof(REAL) * n), *hh = malloc(sizeof(REAL) * n), *ff = malloc(sizeof(REAL) * n);
  int i;
  for (i = 0; i < n; i++) vv[i] = (REAL)v[i];
  if (!h_ready || n > h_nl) { free(vv); free(hh); free(ff); return -1; } /* z/zden/zdiv sized nl */
  fvoigt(damp, vv, n, hh, ff);
  for (i = 0; i < n; i++) { h[i] = hh[i]; f[i] = ff[i]; }
  free(vv); free(hh); free(ff);
  return 0;
}

/* mode 0: direct_convolution (zero padding); mode 1: direct_convolution_ic with Ic. */
int pmref_conv(double *x, int n, const double *taps, int mode, double ic) {
  REAL *xx = malloc(sizeof(REAL) * n);
  PRECISION *hh = malloc(sizeof(PRECISION) * n);
  int i;
  if (!h_ready || n > h_nl) { free(xx); free(hh); return -1; }
  for (i = 0; i < n; i++) { xx[i] = (REAL)x[i]; hh[i] = taps[i]; }
  if (mode == 0) direct_convolution(xx, n, hh, n);
  else direct_convolution_ic(xx, n, hh, n, (REAL)ic);
  for (i = 0; i < n; i++) x[i] = xx[i];
  free(xx); free(hh);
  return 0;
}

/* covarm2 + fchisqr on caller data (sig = per-point variance, 4*nl). */
int pmref_normal_equations(const double *w, const double *sig, const float *spectro, const double *syn,
                           const double *dsyn, double *beta, double *alpha, double nfree, double *chisq) {
  int n4 = h_nl * NPARMS, i;
  REAL ww[4], *sg = malloc(sizeof(REAL) * n4), *sy = malloc(sizeof(REAL) * n4);
  REAL *ds = malloc(sizeof(REAL) * n4 * NTERMS), *bt = malloc(sizeof(REAL) * NTERMS);
  REAL *al = malloc(sizeof(REAL) * NTERMS * NTERMS);
  for (i = 0; i < 4; i++) ww[i] = (REAL)w[i];
  for (i = 0; i < n4; i++) { sg[i] = (REAL)sig[i]; sy[i] = (REAL)syn[i]; }
  for (i = 0; i < n4 * NTERMS; i++) ds[i] = (REAL)dsyn[i];
  covarm2(ww, sg, (float *)spectro, h_nl, sy, ds, bt, al);
  for (i = 0; i < NTERMS; i++) beta[i] = bt[i];
  for (i = 0; i < NTERMS * NTERMS; i++) alpha[i] = al[i];
  if (chisq) *chisq = fchisqr(sy, h_nl, (float *)spectro, ww, sg, (REAL)nfree);
  free(sg); free(sy); free(ds); free(bt); free(al);
  return 0;
}

/* mil_svd on a caller matrix (NTERMS x NTERMS, destroyed like the original). */
int pmref_svd_solve(double *h, const double *beta, double *delta) {
  REAL *bt = malloc(sizeof(REAL) * NTERMS);
  int i;
  for (i = 0; i < NTERMS; i++) bt[i] = (REAL)beta[i];
  mil_svd(h, bt, delta);
  free(bt);
  return 0;
}

/* fgauss_WL (fgauss.c:79-154) into caller storage. */
int pmref_fgauss_wl(double fwhm_ma, double step, double lambda_first, double lambda_central, int n, double *out) {
  int sz = 0, i;
  PRECISION *g = fgauss_WL(fwhm_ma, step, lambda_first, lambda_central, n, &sz);
  for (i = 0; i < sz && i < n; i++) out[i] = g[i];
  free(g);
  return sz;
}

/* interpolationLinearPSF (milosUtils.c:684-738) into caller storage. */
int pmref_interp_psf(const double *dl, const double *psf, int nsamp, const double *offsets, int n,
                     double offset, double *out) {
  int i;
  for (i = 0; i < n; i++) out[i] = 0.0;
  return interpolationLinearPSF((PRECISION *)dl, (PRECISION *)psf, (PRECISION *)offsets, (size_t)nsamp, out,
                                (size_t)n, offset);
}
