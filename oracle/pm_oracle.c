/*
 * pm_oracle.c -- CPU restatement of the P-MILOS per-pixel ME inversion.
 *
 * TEST INFRASTRUCTURE ONLY (see pm_oracle.h).  This is an independent restatement
 * written for this project from the reference's behaviour; every function cites
 * the reference file:line it follows.  Where the reference's result depends on
 * an intermediate being rounded to REAL (float in the default build), this code
 * rounds at the same point, so that the float build agrees bit for bit with the
 * reference compiled under the same flags; the structure is otherwise this
 * project's own (one context struct instead of ~60 process globals, one fused
 * pass per wavelength instead of one loop per intermediate).
 *
 * Macroturbulence follows the reference's direct-convolution branch (a
 * Gaussian correlated with the PSF, then a circular convolution of every
 * profile); the FFT convolution path is out of scope.
 *
 * Response-function rows from 9 up are, as in the reference, never cleared: a
 * row the current call does not write (the macroturbulence row while
 * v_mac <= 1e-4) keeps what an earlier call of the same context left there.
 */
#include "pm_oracle.h"
#include "pm_jacobi.h"
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef PMO_DOUBLE
typedef double real;
#define RSIN(x) sin(x)
#define RCOS(x) cos(x)
#define RSQRT(x) sqrt(x)
#define RFABS(x) fabs(x)
#else
typedef float real;
#define RSIN(x) sinf(x)
#define RCOS(x) cosf(x)
#define RSQRT(x) sqrtf(x)
#define RFABS(x) fabsf(x)
#endif

#define PMO_PI 3.14159265358979323846264338327950288419716939937510
#define PMO_VLIGHT 2.99792458e+5      /* km/s, defines.h:74 */
#define PMO_ZEEMAN 4.6686411e-13      /* e/(4 pi m c^2) in A^-1 G^-1, defines.h:76 */
#define PMO_RSQRTPI 0.5641895836      /* 1/sqrt(pi) as the reference writes it, defines.h:72 */
#define PMO_NCOMP 16                  /* max Zeeman components per group */
#define PMO_GHOST_SIGMA 1000000000000000000000.0 /* milosUtils.c:486 */

enum { I_ETA0 = 0, I_B, I_VLOS, I_DOPP, I_AA, I_GM, I_AZ, I_S0, I_S1, I_MAC, I_ALFA };

typedef struct {
  int n;              /* components in the group */
  real we[PMO_NCOMP]; /* strengths (WEP/WEB/WER) */
  real nu[PMO_NCOMP]; /* splitting in Lande units (NUP/NUB/NUR) */
} zgroup;

/* Per-wavelength quantities that the synthesis leaves behind for the response
 * functions (the reference keeps them in process globals, mil_sinrf.c:18-29). */
typedef struct {
  real fi[3], shi[3];          /* absorption / dispersion profile per group: pi, blue, red */
  real uu[3], H[3], F[3];      /* last component's shifted u, Voigt H and F per group */
  real parcial1, parcial2, parcial3;
  real etain, etaqn, etaun, etavn, rhoqn, rhoun, rhovn;
  real etai, etai_2, gp1, gp2, gp3, dt, dti, g4, g5, g6;
} lam_state;

struct pmo_ctx {
  int nl, K;
  double lambda0;
  double *lambda;
  int has_psf;
  double *psf;
  double *pad; /* 2*nl+1 zero-padded correlation buffer */
  zgroup grp[3];  /* 0 = pi (central), 1 = blue (sigma b), 2 = red (sigma r) */
  real gl, gu, geff, fo;
  /* angle terms of the current synthesis (mil_sinrf.c:84-103) */
  real cc, cc_2;
  real sin_gm, cosi, sinis, cosis, cosis_2, sina, cosa, sinda, cosda, sindi, cosdi, sinis_cosa, sinis_sina;
  real shift[3][PMO_NCOMP]; /* nupB, nubB, nurB (mil_sinrf.c:153-166) */
  lam_state *ls;
  real *spectra, *spectra_slight, *d_spectra, *vsigma, *slight;
  real *spectra_mac;   /* synthesis before any convolution (mil_sinrf.c:278-283) */
  double *gmac, *gmacd; /* macroturbulence kernel and its derivative (GMAC, GMAC_DERIV) */
  real *circ;          /* circular-convolution result buffer (resultConv) */
};

int pmo_sizeof_real(void) { return (int)sizeof(real); }

/* ------------------------------------------------------------------ */
/* Zeeman pattern: Cuanten, create_cuantic.c:60-294.                   */
/* ------------------------------------------------------------------ */
static int zeeman_pattern(pmo_ctx *c, double sl, double ll, double jl, double su, double lu, double ju,
                          double fos) {
  real g1, g2, geff, sum;
  int nlo = (int)(2 * jl + 1), nup = (int)(2 * ju + 1);
  int jj = (int)(ju - jl);
  int n_pi = (int)(2 * (jl < ju ? jl : ju) + 1);
  int n_sig = (int)(jl + ju);
  int a, b, k;
  real wp[PMO_NCOMP], wb[PMO_NCOMP], wr[PMO_NCOMP];
  real mp[PMO_NCOMP], mb[PMO_NCOMP], mr[PMO_NCOMP];
  int ip = 0, ib = 0, ir = 0;
  if (n_pi > PMO_NCOMP || n_sig > PMO_NCOMP || n_pi < 1 || n_sig < 1) return -1;
  /* Lande factors (create_cuantic.c:71-81) */
  g1 = (jl != 0) ? (real)((3.0 * jl * (jl + 1) + sl * (sl + 1) - ll * (ll + 1)) / (2 * jl * (jl + 1))) : 0;
  g2 = (ju != 0) ? (real)((3.0 * ju * (ju + 1.0) + su * (su + 1.0) - lu * (lu + 1.0)) / (2.0 * ju * (ju + 1.0))) : 0;
  geff = (real)((g1 + g2) / 2 + (g1 - g2) * (jl * (jl + 1.) - ju * (ju + 1.)) / 4);
  /* magnetic sublevel pairs (create_cuantic.c:118-184); M_lo = a - jl, M_up = b - ju */
  for (a = 0; a < nlo; a++) {
    int m1 = a - (int)jl;
    for (b = 0; b < nup; b++) {
      int m2 = b - (int)ju;
      int dm = m2 - m1;
      if (dm == 0) {
        wp[ip] = (jj == -1) ? (real)(jl * jl - m1 * m1) : (jj == 0) ? (real)(m1 * m1) : (real)((jl + 1) * (jl + 1) - m1 * m1);
        mp[ip++] = g1 * m1 - g2 * m2;
      } else if (dm == 1) {
        wb[ib] = (jj == -1) ? (real)((jl - m1) * (jl - m1 - 1) / 4) : (jj == 0) ? (real)((jl - m1) * (jl + m1 + 1) / 4) : (real)((jl + m1 + 1) * (jl + m1 + 2) / 4);
        mb[ib++] = g1 * m1 - g2 * m2;
      } else if (dm == -1) {
        wr[ir] = (jj == -1) ? (real)((jl + m1) * (jl + m1 - 1) / 4) : (jj == 0) ? (real)((jl + m1) * (jl - m1 + 1) / 4) : (real)((jl - m1 + 1) * (jl - m1 + 2) / 4);
        mr[ir++] = g1 * m1 - g2 * m2;
      }
    }
  }
  if (ip != n_pi || ib != n_sig || ir != n_sig) return -2;
  /* normalise each group to unit total strength (create_cuantic.c:186-218) */
  sum = 0; for (k = 0; k < n_pi; k++) sum = sum + wp[k];
  for (k = 0; k < n_pi; k++) wp[k] = wp[k] / sum;
  sum = 0; for (k = 0; k < n_sig; k++) sum = sum + wb[k];
  for (k = 0; k < n_sig; k++) wb[k] = wb[k] / sum;
  sum = 0; for (k = 0; k < n_sig; k++) sum = sum + wr[k];
  for (k = 0; k < n_sig; k++) wr[k] = wr[k] / sum;
  c->grp[0].n = n_pi; c->grp[1].n = n_sig; c->grp[2].n = n_sig;
  for (k = 0; k < n_pi; k++) { c->grp[0].we[k] = wp[k]; c->grp[0].nu[k] = mp[k]; }
  for (k = 0; k < n_sig; k++) {
    c->grp[1].we[k] = wb[k]; c->grp[1].nu[k] = mb[k];
    c->grp[2].we[k] = wr[k]; c->grp[2].nu[k] = mr[k];
  }
  c->gl = g1; c->gu = g2; c->geff = geff; c->fo = (real)fos;
  return 0;
}

pmo_ctx *pmo_create(int nlambda, const double *lambda, double lambda0, const double *cuantic_dat,
                    const double *psf, int nterms) {
  pmo_ctx *c;
  int i;
  if (nlambda < 2 || nterms < 1 || nterms > 11) return NULL;
  c = (pmo_ctx *)calloc(1, sizeof(pmo_ctx));
  c->nl = nlambda;
  c->K = nterms;
  c->lambda0 = lambda0;
  c->lambda = (double *)malloc(sizeof(double) * nlambda);
  for (i = 0; i < nlambda; i++) c->lambda[i] = lambda[i];
  c->has_psf = psf != NULL;
  c->psf = (double *)calloc(nlambda, sizeof(double));
  if (psf) for (i = 0; i < nlambda; i++) c->psf[i] = psf[i];
  c->pad = (double *)calloc(2 * nlambda + 1, sizeof(double));
  c->ls = (lam_state *)calloc(nlambda, sizeof(lam_state));
  c->spectra = (real *)calloc(4 * nlambda, sizeof(real));
  c->spectra_slight = (real *)calloc(4 * nlambda, sizeof(real));
  c->d_spectra = (real *)calloc(4 * nlambda * nterms, sizeof(real));
  c->vsigma = (real *)calloc(4 * nlambda, sizeof(real));
  c->slight = (real *)calloc(4 * nlambda, sizeof(real));
  c->spectra_mac = (real *)calloc(4 * nlambda, sizeof(real));
  c->gmac = (double *)calloc(nlambda, sizeof(double));
  c->gmacd = (double *)calloc(nlambda, sizeof(double));
  c->circ = (real *)calloc(nlambda, sizeof(real));
  /* milos.c:232-233 */
  c->cc = (real)(PMO_PI / 180.0);
  c->cc_2 = c->cc * 2;
  if (zeeman_pattern(c, cuantic_dat[1], cuantic_dat[2], cuantic_dat[3], cuantic_dat[4], cuantic_dat[5],
                     cuantic_dat[6], 1.0) != 0) {
    pmo_destroy(c);
    return NULL;
  }
  return c;
}

void pmo_destroy(pmo_ctx *c) {
  if (!c) return;
  free(c->lambda); free(c->psf); free(c->pad); free(c->ls);
  free(c->spectra); free(c->spectra_slight); free(c->d_spectra); free(c->vsigma); free(c->slight);
  free(c->spectra_mac); free(c->gmac); free(c->gmacd); free(c->circ);
  free(c);
}

int pmo_cuantic(const pmo_ctx *c, double *out, int cap) {
  int k = 0, i, np = c->grp[0].n, ns = c->grp[1].n;
  if (cap < 6 + 4 * ns + 2 * np) return -2;
  out[k++] = np; out[k++] = ns; out[k++] = c->gl; out[k++] = c->gu; out[k++] = c->geff; out[k++] = c->fo;
  for (i = 0; i < ns; i++) out[k++] = c->grp[1].nu[i];
  for (i = 0; i < np; i++) out[k++] = c->grp[0].nu[i];
  for (i = 0; i < ns; i++) out[k++] = c->grp[2].nu[i];
  for (i = 0; i < ns; i++) out[k++] = c->grp[1].we[i];
  for (i = 0; i < np; i++) out[k++] = c->grp[0].we[i];
  for (i = 0; i < ns; i++) out[k++] = c->grp[2].we[i];
  return k;
}

/* ------------------------------------------------------------------ */
/* Voigt and Faraday-Voigt profiles: fvoigt.c:15-80.                   */
/* Hui, Armstrong & Wray (1978) rational approximation of the complex  */
/* probability function w(z), z = a - i v: numerator of degree 6,      */
/* monic denominator of degree 7, evaluated by Horner's rule in double */
/* complex arithmetic.  H = Re w, F = Im w / 2.  The coefficient table */
/* is the published one and must equal the reference's for parity.     */
/* ------------------------------------------------------------------ */
static const double hui_p[7] = {122.607931777104326, 214.382388694706425, 181.928533092181549,
                                93.155580458138441,  30.180142196210589,  5.912626209773153,
                                0.564189583562615};
static const double hui_q[8] = {122.60793177387535, 352.730625110963558, 457.334478783897737,
                                348.703917719495792, 170.354001821091472, 53.992906912940207,
                                10.479857114260399, 1.};

static void voigt1(double damp, real v, real *h, real *f) {
  double _Complex z = damp - v * _Complex_I;
  double _Complex num = hui_p[6], den = z + hui_q[6], w;
  int j;
  for (j = 5; j >= 0; j--) num = num * z + hui_p[j];
  for (j = 5; j >= 0; j--) den = den * z + hui_q[j];
  w = num / den;
  *h = (real)creal(w);
  *f = (real)((double)cimag(w) * 0.5);
}

int pmo_fvoigt(double damp, const double *v, int n, double *h, double *f) {
  int i;
  for (i = 0; i < n; i++) {
    real hh, ff;
    voigt1(damp, (real)v[i], &hh, &ff);
    h[i] = hh;
    f[i] = ff;
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* Instrumental profile: direct correlation with the nl-tap kernel     */
/* centred at nl/2, convolution.c:54-121.  mode 0: zero padding (Q,U,V */
/* and the Q,U,V response functions); mode 1: correlate Ic - x and     */
/* return Ic - result, i.e. pad with the continuum (Stokes I).          */
/* Accumulation in double, as the reference does.                      */
/* ------------------------------------------------------------------ */
static void correlate(const pmo_ctx *c, real *x, int with_ic, real ic) {
  const int n = c->nl, half = n / 2;
  int k, j;
  for (k = 0; k < n; k++) c->pad[k + half] = with_ic ? (double)(ic - x[k]) : (double)x[k];
  for (k = 0; k < n; k++) {
    double acc = 0;
    for (j = 0; j < n; j++) acc += c->psf[j] * c->pad[j + k];
    x[k] = with_ic ? (real)((double)ic - acc) : (real)acc;
  }
}

static real edge_max(const real *x, int n) { return (x[0] > x[n - 1]) ? x[0] : x[n - 1]; }

/* The same correlation of a double kernel with the PSF, direct_convolution_double
 * (convolution.c:21-42): the macroturbulence kernel seen through the instrument. */
static void correlate_d(const pmo_ctx *c, double *x) {
  const int n = c->nl, half = n / 2;
  int k, j;
  for (k = 0; k < n; k++) c->pad[k + half] = x[k];
  for (k = 0; k < n; k++) {
    double acc = 0;
    for (j = 0; j < n; j++) acc += c->psf[j] * c->pad[j + k];
    x[k] = acc;
  }
}

/* ------------------------------------------------------------------ */
/* Macroturbulence.  fgauss (fgauss.c:16-66): a Gaussian over the grid, */
/* centred at lambda[nl/2], of sigma = lambda0 v_mac / c, normalised to */
/* unit sum; its derivative w.r.t. v_mac as me_der.c:419-421 forms it.   */
/* convCircular (convolution.c:125-153): y[i] = sum_j h[j] x[(i-j) mod  */
/* n] in double, stored rotated by nl/2 (result[m] = y[(m + nl/2) mod   */
/* n]) and rounded to REAL.                                             */
/* ------------------------------------------------------------------ */
static void mac_kernel(const pmo_ctx *c, double mac, double *g, double *gd) {
  const int n = c->nl;
  const double centre = c->lambda[n / 2];
  const double ild = (c->lambda0 * mac) / PMO_VLIGHT;
  double cte = 0;
  int i;
  for (i = 0; i < n; i++) {
    const double a = (c->lambda[i] - centre) / ild;
    const double term = (a * a) / 2;
    g[i] = (term < 1e30) ? exp(-term) : 0;
  }
  for (i = 0; i < n; i++) cte += g[i];
  for (i = 0; i < n; i++) g[i] /= cte;
  if (gd)
    for (i = 0; i < n; i++) {
      const double a = (c->lambda[i] - centre) / ild;
      gd[i] = g[i] / mac * (a * a - 1.0);
    }
}

static void circular(const pmo_ctx *c, const real *x, const double *h, real *out) {
  const int n = c->nl, half = n / 2;
  int i, j;
  for (i = 0; i < n; i++) {
    double acc = 0;
    for (j = 0; j < n; j++) acc += h[j] * x[(i - j + n) % n];
    c->circ[(i - half + n) % n] = (real)acc;
  }
  for (i = 0; i < n; i++) out[i] = c->circ[i];
}

int pmo_conv(const pmo_ctx *c, double *x, int mode, double ic) {
  real *t = (real *)malloc(sizeof(real) * c->nl);
  int i;
  for (i = 0; i < c->nl; i++) t[i] = (real)x[i];
  correlate(c, t, mode == 1, (real)ic);
  for (i = 0; i < c->nl; i++) x[i] = t[i];
  free(t);
  return 0;
}

/* ------------------------------------------------------------------ */
/* ME synthesis: mil_sinrf.c:46-415 (single line).                     */
/* ------------------------------------------------------------------ */
static int synthesis(pmo_ctx *c, const double *m, real ah, const real *slight) {
  const int n = c->nl;
  const double E00 = m[I_ETA0], MF = m[I_B], VL = m[I_VLOS], LD = m[I_DOPP], A = m[I_AA];
  const double B0 = m[I_S0], B1 = -((m[I_S1]) * ah), ALF = m[I_ALFA];
  double AZI, GM, E0;
  real ulos, parcial, E0_2, cosi_E0_2;
  int i, g, k;
  const int mac_on = m[I_MAC] > 0.0001;
  if (mac_on && c->K < 10) return -3; /* v_mac > 0 needs its RF row (NTERMS >= 10, milos.c:152-157) */

  /* angle terms, mil_sinrf.c:84-103 */
  AZI = m[I_AZ] * c->cc;
  GM = m[I_GM] * c->cc;
  c->sin_gm = RSIN((real)GM);
  c->cosi = RCOS((real)GM);
  c->sinis = c->sin_gm * c->sin_gm;
  c->cosis = c->cosi * c->cosi;
  c->cosis_2 = (1 + c->cosis) / 2;
  {
    real azi_2 = (real)(2 * AZI);
    c->sina = RSIN(azi_2);
    c->cosa = RCOS(azi_2);
  }
  c->sinda = c->cosa * c->cc_2;
  c->cosda = -c->sina * c->cc_2;
  c->sindi = c->cosi * c->sin_gm * c->cc_2;
  c->cosdi = -c->sin_gm * c->cc;
  c->sinis_cosa = c->sinis * c->cosa;
  c->sinis_sina = c->sinis * c->sina;

  /* line strength, Doppler shift and Zeeman splitting, mil_sinrf.c:117-166 */
  E0 = E00 * c->fo;
  ulos = (real)((VL * c->lambda0) / (PMO_VLIGHT * LD));
  parcial = (real)(((c->lambda0 * c->lambda0) / LD) * PMO_ZEEMAN);
  for (k = 0; k < c->grp[1].n; k++) c->shift[1][k] = parcial * c->grp[1].nu[k];
  for (k = 0; k < c->grp[0].n; k++) c->shift[0][k] = parcial * c->grp[0].nu[k];
  for (k = 0; k < c->grp[2].n; k++) c->shift[2][k] = -c->shift[1][c->grp[1].n - (k + 1)];
  E0_2 = (real)(E0 / 2.0);
  cosi_E0_2 = E0_2 * c->cosi;

  for (i = 0; i < n; i++) {
    lam_state *s = &c->ls[i];
    real u = (real)(((c->lambda[i] - c->lambda0) / LD) - ulos);
    real etaq, etau, etav, rhoq, rhou, rhov, auxq, auxu, auxv, gp4, gp5, gp6, dtiaux;
    /* absorption/dispersion profiles of the three groups, funcionComponentFor_sinrf
     * (mil_sinrf.c:418-449): sum of strength-weighted Voigt/Faraday profiles */
    for (g = 0; g < 3; g++) {
      real fi = 0, shi = 0;
      for (k = 0; k < c->grp[g].n; k++) {
        real uu = (real)(u - c->shift[g][k] * MF), H, F;
        voigt1(A, uu, &H, &F);
        fi = fi + c->grp[g].we[k] * H;
        shi = (shi + (c->grp[g].we[k] * F * 2));
        s->uu[g] = uu; s->H[g] = H; s->F[g] = F;
      }
      s->fi[g] = fi;
      s->shi[g] = shi;
    }
    /* propagation matrix elements, mil_sinrf.c:191-223 */
    s->parcial1 = s->fi[1] + s->fi[2];
    s->parcial2 = (E0_2) * (s->fi[0] - (s->parcial1) / 2);
    s->parcial3 = (E0_2) * (s->shi[0] - (s->shi[1] + s->shi[2]) / 2);
    s->etain = ((E0_2) * (s->fi[0] * c->sinis + (s->parcial1) * c->cosis_2));
    s->etaqn = (s->parcial2 * c->sinis_cosa);
    s->etaun = (s->parcial2 * c->sinis_sina);
    s->etavn = (s->fi[2] - s->fi[1]) * cosi_E0_2;
    s->rhoqn = (s->parcial3 * c->sinis_cosa);
    s->rhoun = (s->parcial3 * c->sinis_sina);
    s->rhovn = (s->shi[2] - s->shi[1]) * cosi_E0_2;
    s->etai = (real)(1.0 + s->etain);
    etaq = s->etaqn; etau = s->etaun; etav = s->etavn;
    rhoq = s->rhoqn; rhou = s->rhoun; rhov = s->rhovn;
    /* Unno-Rachkovsky solution of the ME atmosphere, mil_sinrf.c:229-285 */
    s->etai_2 = s->etai * s->etai;
    auxq = rhoq * rhoq; auxu = rhou * rhou; auxv = rhov * rhov;
    s->gp1 = s->etai_2 - etaq * etaq - etau * etau - etav * etav + auxq + auxu + auxv;
    s->gp3 = s->etai_2 + auxq + auxu + auxv;
    s->gp2 = etaq * rhoq + etau * rhou + etav * rhov;
    s->dt = s->etai_2 * s->gp1 - s->gp2 * s->gp2;
    s->dti = (real)(1.0 / s->dt);
    gp4 = s->etai_2 * etaq + s->etai * (etav * rhou - etau * rhov);
    gp5 = s->etai_2 * etau + s->etai * (etaq * rhov - etav * rhoq);
    gp6 = (s->etai_2) * etav + s->etai * (etau * rhoq - etaq * rhou);
    s->g4 = gp4 + rhoq * s->gp2;
    s->g5 = gp5 + rhou * s->gp2;
    s->g6 = gp6 + rhov * s->gp2;
    dtiaux = (real)(s->dti * (B1));
    c->spectra[i] = (real)(B0 - dtiaux * s->etai * s->gp3);
    c->spectra[i + n] = (dtiaux * (s->g4));
    c->spectra[i + 2 * n] = (dtiaux * (s->g5));
    c->spectra[i + 3 * n] = (dtiaux * (s->g6));
    for (k = 0; k < 4; k++) c->spectra_mac[i + k * n] = c->spectra[i + k * n];
  }

  if (mac_on) {
    /* macroturbulence (mil_sinrf.c:288-357, direct branch): the PSF folds into
     * the Gaussian, and every profile, I included, is convolved circularly */
    mac_kernel(c, m[I_MAC], c->gmac, NULL);
    if (c->has_psf) correlate_d(c, c->gmac);
    for (k = 0; k < 4; k++) circular(c, c->spectra + k * n, c->gmac, c->spectra + k * n);
  } else if (c->has_psf) {
    /* instrumental profile, mil_sinrf.c:387-402 */
    correlate(c, c->spectra, 1, edge_max(c->spectra, n));
    for (k = 1; k < 4; k++) correlate(c, c->spectra + k * n, 0, 0);
  }
  /* stray-light mix, mil_sinrf.c:405-412 */
  if (slight) {
    for (i = 0; i < 4 * n; i++) {
      c->spectra_slight[i] = c->spectra[i];
      c->spectra[i] = (real)(c->spectra[i] * ALF + slight[i] * (1.0 - ALF));
    }
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* Analytic response functions: me_der.c:48-530 and funcionComponentFor */
/* me_der.c:536-609.  Must follow a synthesis at the same model.  The   */
/* RF layout is d[(s*K + k)*nl + i] (Stokes s, parameter k, lambda i).  */
/* ff_spectra is the spectrum the filling-factor RF is built from: the  */
/* unmixed synthesis on the first call of lm_mils, the stray-light-     */
/* mixed one after an accepted step (milosUtils.c:537 vs :587).         */
/* ------------------------------------------------------------------ */
static void response_functions(pmo_ctx *c, const double *m, real ah, const real *slight, const real *ff_spectra,
                               const int *fix) {
  const int n = c->nl, K = c->K;
  const double E00 = m[I_ETA0], LD = m[I_DOPP], A = m[I_AA], B1 = -((m[I_S1]) * ah), ALF = m[I_ALFA];
  const double E0 = E00 * c->fo;
  real *d = c->d_spectra;
  real auxCte, E0_2, sc, ss, sindi_cosa, sindi_sina, cosdi_E0_2, cosi_2_E0, cosis_2_E0_2, sinis_E0_2;
  real cosi_cosdi, sindi_E0_2, sinis_cosda, sinis_sinda;
  int i, k, s, g, il;

  auxCte = (real)((-c->lambda0) / (PMO_VLIGHT * LD));
  /* me_der.c:118-127: the angle products are rescaled in place by E0/2 */
  sc = (real)(E0 * c->sinis_cosa / 2);
  ss = (real)(E0 * c->sinis_sina / 2);
  E0_2 = (real)(E0 / 2.0);
  sindi_cosa = c->sindi * c->cosa;
  sindi_sina = c->sindi * c->sina;
  cosdi_E0_2 = (E0_2) * c->cosdi;
  cosi_2_E0 = (real)(E0 * c->cosi / 2.0);
  cosis_2_E0_2 = c->cosis_2 * E0_2;
  sinis_E0_2 = c->sinis * E0_2;
  cosi_cosdi = c->cosi * c->cosdi * E0_2;
  sindi_E0_2 = c->sindi * E0_2;
  sinis_cosda = c->sinis * c->cosda;
  sinis_sinda = c->sinis * c->sinda;

  for (i = 0; i < n; i++) {
    const lam_state *st = &c->ls[i];
    /* derivatives of the group profiles w.r.t. B, vlos, dopp, a; per group only the
     * last component's terms survive, as in the reference (me_der.c:569-600
     * assigns rather than accumulates) */
    real dfi[3][4], dshi[3][4];
    real de[7], dq[7], du[7], dv[7], rq[7], ru[7], rv[7];
    real etai = st->etai, etai_2 = st->etai_2, etaq = st->etaqn, etau = st->etaun, etav = st->etavn;
    real rhoq = st->rhoqn, rhou = st->rhoun, rhov = st->rhovn;
    real dtaux, etai_gp3, aux2e, ext1, ext2, ext3, ext4, dti_s1;
    for (g = 0; g < 3; g++) {
      int last = c->grp[g].n - 1;
      real we = c->grp[g].we[last], nu = c->shift[g][last];
      real uu = st->uu[g], H = st->H[g], F = st->F[g];
      real dH_u = (real)(((4 * A * F) - (2 * uu * H)) * we);
      real dF_u = (real)((PMO_RSQRTPI - A * H - 2 * uu * F) * we);
      real uun = (real)(-uu / LD);
      dfi[g][0] = dH_u * (-nu);
      dfi[g][1] = dH_u * auxCte;
      dfi[g][2] = (dH_u * uun);
      dfi[g][3] = (-2 * dF_u);
      dshi[g][0] = (dF_u) * (-nu);
      dshi[g][1] = dF_u * auxCte;
      dshi[g][2] = (dF_u * uun);
      dshi[g][3] = (dH_u / 2);
    }
    /* eta0: me_der.c:93-113 */
    de[0] = (real)(st->etain / E0);
    dq[0] = (real)(st->etaqn / E0);
    du[0] = (real)(st->etaun / E0);
    dv[0] = (real)(st->etavn / E0);
    rq[0] = (real)(st->rhoqn / E0);
    ru[0] = (real)(st->rhoun / E0);
    rv[0] = (real)(st->rhovn / E0);
    /* B, vlos, dopp, a: me_der.c:130-154 */
    for (k = 1; k < 5; k++) {
      real dfisum = dfi[1][k - 1] + dfi[2][k - 1];
      real aux = dfi[0][k - 1] - dfisum / 2;
      real auxr;
      de[k] = (dfi[0][k - 1] * sinis_E0_2 + dfisum * cosis_2_E0_2);
      dq[k] = (aux) * sc;
      du[k] = (aux) * ss;
      dv[k] = (dfi[2][k - 1] - dfi[1][k - 1]) * cosi_2_E0;
      auxr = (real)(dshi[0][k - 1] - (dshi[1][k - 1] + dshi[2][k - 1]) / 2.0);
      rq[k] = (auxr) * sc;
      ru[k] = (auxr) * ss;
      rv[k] = ((dshi[2][k - 1] - dshi[1][k - 1])) * cosi_2_E0;
    }
    /* gamma: me_der.c:157-180 */
    de[5] = st->fi[0] * sindi_E0_2 + (st->parcial1) * cosi_cosdi;
    dq[5] = st->parcial2 * sindi_cosa;
    du[5] = st->parcial2 * sindi_sina;
    dv[5] = (st->fi[2] - st->fi[1]) * cosdi_E0_2;
    rq[5] = st->parcial3 * sindi_cosa;
    ru[5] = st->parcial3 * sindi_sina;
    rv[5] = (st->shi[2] - st->shi[1]) * cosdi_E0_2;
    /* azimuth: me_der.c:183-199 (eta_I, eta_V, rho_V do not depend on it) */
    de[6] = 0; dv[6] = 0; rv[6] = 0;
    dq[6] = st->parcial2 * sinis_cosda;
    du[6] = st->parcial2 * sinis_sinda;
    rq[6] = st->parcial3 * sinis_cosda;
    ru[6] = st->parcial3 * sinis_sinda;

    /* chain rule through the ME solution, me_der.c:207-277 */
    dtaux = (real)((B1) / (st->dt * st->dt));
    etai_gp3 = etai * st->gp3;
    aux2e = 2 * etai;
    ext1 = aux2e * etaq + etav * rhou - etau * rhov;
    ext2 = aux2e * etau + etaq * rhov - etav * rhoq;
    ext3 = aux2e * etav + etau * rhoq - etaq * rhou;
    ext4 = aux2e * st->gp1;
    for (il = 0; il < 7; il++) {
      real dgp1 = (real)(2.0 * (etai * de[il] - etaq * dq[il] - etau * du[il] - etav * dv[il] + rhoq * rq[il] +
                                rhou * ru[il] + rhov * rv[il]));
      real dgp2 = rhoq * dq[il] + etaq * rq[il] + rhou * du[il] + etau * ru[il] + rhov * dv[il] + etav * rv[il];
      real d_dt = ext4 * de[il] + etai_2 * dgp1 - 2 * st->gp2 * dgp2;
      real dgp3 = (real)(2.0 * (etai * de[il] + rhoq * rq[il] + rhou * ru[il] + rhov * rv[il]));
      real dgp4, dgp5, dgp6;
      d[i + n * il] = -(((de[il] * st->gp3 + etai * dgp3) * st->dt - d_dt * etai_gp3) * (dtaux));
      dgp4 = de[il] * (ext1) + (etai_2) * dq[il] + etai * (rhou * dv[il] + etav * ru[il] - rhov * du[il] - etau * rv[il]);
      d[i + n * il + n * K] = ((dgp4 + rq[il] * st->gp2 + rhoq * dgp2) * st->dt - d_dt * (st->g4)) * (dtaux);
      dgp5 = de[il] * (ext2) + (etai_2) * du[il] + etai * (rhov * dq[il] + etaq * rv[il] - rhoq * dv[il] - etav * rq[il]);
      d[i + n * il + (n * K * 2)] = ((dgp5 + ru[il] * st->gp2 + rhou * dgp2) * st->dt - d_dt * (st->g5)) * (dtaux);
      dgp6 = de[il] * (ext3) + (etai_2) * dv[il] + etai * (rhoq * du[il] + etau * rq[il] - rhou * dq[il] - etaq * ru[il]);
      d[i + n * il + (n * K * 3)] = ((dgp6 + rv[il] * st->gp2 + rhov * dgp2) * st->dt - d_dt * (st->g6)) * (dtaux);
    }
    /* S1 and S0, me_der.c:281-306; azimuth I and V vanish, :309-312 */
    dti_s1 = -(st->dti * ah);
    d[i + n * 8] = -dti_s1 * etai_gp3;
    d[i + n * 8 + (n * K)] = dti_s1 * (st->g4);
    d[i + n * 8 + (n * K * 2)] = dti_s1 * (st->g5);
    d[i + n * 8 + (n * K * 3)] = dti_s1 * (st->g6);
    d[i + n * 7] = 1;
    d[i + n * 7 + (n * K)] = 0;
    d[i + n * 7 + (n * K * 2)] = 0;
    d[i + n * 7 + (n * K * 3)] = 0;
    d[i + n * 6] = 0;
    d[i + n * 6 + (n * K * 3)] = 0;
  }

  if (m[I_MAC] > 0.0001 && K >= 10) {
    /* macroturbulence, me_der.c:314-438 (direct branch): row 9 is the circular
     * convolution of the unconvolved synthesis with the kernel's derivative,
     * rows 0..8 but S0 are convolved circularly with the kernel; both kernels
     * pass through the PSF first */
    mac_kernel(c, m[I_MAC], c->gmac, c->gmacd);
    if (c->has_psf) {
      correlate_d(c, c->gmacd);
      correlate_d(c, c->gmac);
    }
    for (s = 0; s < 4; s++) circular(c, c->spectra_mac + n * s, c->gmacd, d + 9 * n + n * K * s);
    for (s = 0; s < 4; s++)
      for (k = 0; k < 9; k++)
        if (k != 7) circular(c, d + n * k + n * K * s, c->gmac, d + n * k + n * K * s);
  } else if (c->has_psf) {
    /* instrumental profile on every RF but S0's, me_der.c:471-496 */
    for (k = 0; k < K; k++)
      if (k != 7) correlate(c, d + n * k, 1, edge_max(d + n * k, n));
    for (s = 1; s < 4; s++)
      for (k = 0; k < K; k++)
        if (k != 7) correlate(c, d + n * k + n * K * s, 0, 0);
  }
  /* filling factor: scale every RF by alpha and build dS/dalpha = S_mag - S_stray,
   * me_der.c:499-525 */
  if (slight) {
    for (s = 0; s < 4; s++)
      for (k = 0; k < K; k++)
        for (i = 0; i < n; i++) {
          real *p = &d[(n * k + n * K * s) + i];
          *p = (real)(*p * ALF);
          if ((K == 11 && k == 10) || (K != 11 && ((fix[9] && k == 10) || (!fix[9] && k == 9))))
            *p = ff_spectra[n * s + i] - slight[n * s + i];
        }
  }
}

/* FijaACeroDerivadasNoNecesarias, milosUtils.c:199-227 */
static void zero_fixed_rfs(pmo_ctx *c, const int *fix) {
  const int n = c->nl, K = c->K;
  int k, s, i;
  for (k = 0; k < K; k++) {
    int zero;
    if (K == 10 && k == 9) zero = (fix[9] == 0 && fix[10] == 0);
    else if (K == 9 || K == 11 || K == 10) zero = (fix[k] == 0);
    else zero = 0;
    if (zero)
      for (s = 0; s < 4; s++)
        for (i = 0; i < n; i++) c->d_spectra[i + n * k + s * n * K] = 0;
  }
}

/* ------------------------------------------------------------------ */
/* Normal equations and merit function: covarm2 lib.c:71-116,          */
/* totalParcialf/Matrixf lib.c:237-268, fchisqr lib.c:126-152.          */
/* ------------------------------------------------------------------ */
static void normal_equations(const pmo_ctx *c, const real *w, const real *sig, const float *obs, real *beta,
                             real *alpha) {
  const int n = c->nl, K = c->K;
  real ap[4][11 * 11], bt[4][11];
  int s, a, b, k;
  for (s = 0; s < 4; s++) {
    const real *ds = c->d_spectra + s * n * K;
    for (a = 0; a < K; a++)
      for (b = 0; b < K; b++) {
        real sum = 0, sum2 = 0;
        for (k = 0; k < n; k++) {
          real db = ds[b * n + k];
          sum += (ds[a * n + k] * db) * (w[s] / sig[n * s + k]);
          if (a == 0) {
            real opa = w[s] * (c->spectra[k + n * s] - obs[k + n * s]);
            sum2 += ((opa * db)) / sig[n * s + k];
          }
        }
        ap[s][K * a + b] = sum;
        if (a == 0) bt[s][b] = sum2;
      }
  }
  for (a = 0; a < K; a++) {
    real sum = 0;
    for (s = 0; s < 4; s++) sum += bt[s][a];
    beta[a] = sum;
  }
  for (a = 0; a < K * K; a++) {
    real sum = 0;
    for (s = 0; s < 4; s++) sum += ap[s][a];
    alpha[a] = sum;
  }
}

static real chisq(const pmo_ctx *c, const float *obs, const real *w, const real *sig, real nfree) {
  const int n = c->nl;
  real tot = 0, o[4] = {0, 0, 0, 0};
  int i, s;
  for (i = 0; i < n; i++)
    for (s = 0; s < 4; s++) {
      real dif = c->spectra[i + n * s] - obs[i + n * s];
      o[s] += (((dif * dif) * w[s]) / (sig[i + n * s]));
    }
  tot += o[0] + o[1] + o[2] + o[3];
  return tot / nfree;
}

/* ------------------------------------------------------------------ */
/* Damped solve: mil_svd, milosUtils.c:237-271.                         */
/* ------------------------------------------------------------------ */
static void svd_solve(int K, double *h, const real *beta, double *delta) {
  const double eps = 1e-12;
  double a[11 * 11], w[11], v[11 * 11], aux2[11];
  int i, j;
  /* the eigen-solver reads the diagonal and lower triangle */
  for (i = 0; i < K; i++)
    for (j = 0; j <= i; j++) { a[i * K + j] = h[i * K + j]; a[j * K + i] = h[i * K + j]; }
  pm_jacobi_eigen(a, (size_t)K, w, v);
  for (j = 0; j < K; j++) {
    double sum = 0;
    for (i = 0; i < K; i++) sum += beta[i] * v[i * K + j];
    aux2[j] = sum * ((fabs(w[j]) > eps) ? (1 / w[j]) : 0.0);
  }
  for (i = 0; i < K; i++) {
    double sum = 0;
    for (j = 0; j < K; j++) sum += v[i * K + j] * aux2[j];
    delta[i] = sum;
  }
}

int pmo_svd_solve(int K, double *covar, const double *beta, double *delta) {
  real bt[11];
  int i;
  if (K < 1 || K > 11) return -1;
  for (i = 0; i < K; i++) bt[i] = (real)beta[i];
  svd_solve(K, covar, bt, delta);
  return 0;
}

/* AplicaDelta, milosUtils.c:47-115 (delta is clamped in place, like the original) */
static void apply_delta(const double *m, double *delta, const int *fix, int K, double *out) {
  if (fix[0]) out[I_ETA0] = m[I_ETA0] - delta[0];
  if (fix[1]) {
    if (delta[1] < -300) delta[1] = -300;
    else if (delta[1] > 300) delta[1] = 300;
    out[I_B] = m[I_B] - delta[1];
  }
  if (fix[2]) out[I_VLOS] = m[I_VLOS] - delta[2];
  if (fix[3]) out[I_DOPP] = m[I_DOPP] - delta[3];
  if (fix[4]) out[I_AA] = m[I_AA] - delta[4];
  if (fix[5]) {
    if (delta[5] < -30) delta[5] = -30;
    else if (delta[5] > 30) delta[5] = 30;
    out[I_GM] = m[I_GM] - delta[5];
  }
  if (fix[6]) {
    if (delta[6] < -30) delta[6] = -30;
    else if (delta[6] > 30) delta[6] = 30;
    out[I_AZ] = m[I_AZ] - delta[6];
  }
  if (fix[7]) out[I_S0] = m[I_S0] - delta[7];
  if (fix[8]) out[I_S1] = m[I_S1] - delta[8];
  if (fix[9]) out[I_MAC] = m[I_MAC] - delta[9];
  if (fix[10]) out[I_ALFA] = m[I_ALFA] - delta[K == 11 ? 10 : 9];
}

/* check, milosUtils.c:118-196: fold B < 0 into the inclination, wrap the angles,
 * clamp the physical ranges */
static void clamp_model(double *m) {
  if (m[I_B] < 0) { m[I_B] = -(m[I_B]); m[I_GM] = 180.0 - (m[I_GM]); }
  if (m[I_B] > 5000) m[I_B] = 5000;
  if (m[I_GM] < 0) m[I_GM] = -(m[I_GM]);
  if (m[I_GM] > 180) m[I_GM] = 360.0 - m[I_GM];
  if (m[I_AZ] < 0) m[I_AZ] = 180 + (m[I_AZ]);
  if (m[I_AZ] > 180) m[I_AZ] = m[I_AZ] - 180.0;
  if (m[I_ETA0] < 1) m[I_ETA0] = 1;
  if (m[I_ETA0] > 2500) m[I_ETA0] = 2500;
  if (m[I_VLOS] < (-20)) m[I_VLOS] = (-20);
  if (m[I_VLOS] > 20) m[I_VLOS] = 20;
  if (m[I_DOPP] < 0.0001) m[I_DOPP] = 0.0001;
  if (m[I_DOPP] > 0.6) m[I_DOPP] = 0.6;
  if (m[I_AA] < 0.0001) m[I_AA] = 0.0001;
  if (m[I_AA] > 10.0) m[I_AA] = 10.0;
  if (m[I_S0] < 0.0001) m[I_S0] = 0.0001;
  if (m[I_S0] > 2.00) m[I_S0] = 2.00;
  if (m[I_S1] < 0.0001) m[I_S1] = 0.0001;
  if (m[I_S1] > 2.00) m[I_S1] = 2.00;
  if (m[I_MAC] < 0) m[I_MAC] = 0;
  if (m[I_MAC] > 4) m[I_MAC] = 4;
  if (m[I_ALFA] < 0) m[I_ALFA] = 0.0;
  if (m[I_ALFA] > 1.0) m[I_ALFA] = 1.0;
}

/* ------------------------------------------------------------------ */
/* Classical estimates: estimacionesClasicas, milosUtils.c:287-452.     */
/* Weak-field centre-of-gravity B_los, v_los from the I centroid,       */
/* inclination from sum|V| m / sum V^2, azimuth from the Q,U sums with  */
/* the quadrant rules.  initial_use = forInitialUse: 1 before lm_mils   */
/* (inclinations within 5 deg of 90 kept off it for B, :395-402), 0 in  */
/* the classical-estimates-only mode (S0 = B_los, :449-450).            */
/* ------------------------------------------------------------------ */
static void classical(const pmo_ctx *c, const float *spectro, double *m, int initial_use) {
  const int n = c->nl;
  const double l0 = c->lambda0;
  const float *sI = spectro, *sQ = spectro + n, *sU = spectro + 2 * n, *sV = spectro + 3 * n;
  int begin = 0, end = n, i;
  double x, y, xv, yv, lp, lm, C, Blos, Vlos, Ic, tan_gamma, gamma_rad, gamma, sum_u, sum_q, tan2phi, phi, B_aux;
  /* ghost wavelengths (I < 0) at either end are skipped */
  for (i = 0; i < n && sI[i] < 0; i++) begin++;
  for (i = n - 1; i >= 0 && sI[i] < 0; i--) end--;
  Ic = spectro[end - 1];
  x = y = xv = yv = 0;
  for (i = begin; i < end - 1; i++)
    if (sI[i] > -1 && sV[i] > -1) {
      double a = (Ic - (sI[i] + sV[i])), av = (Ic - sI[i]);
      x += (a * (c->lambda[i] - l0));
      xv += (av * (c->lambda[i] - l0));
      y += a;
      yv += av;
    }
  lp = (fabs(y) > 1e-15) ? x / y : 0;
  x = y = 0;
  for (i = begin; i < end - 1; i++)
    if (sI[i] > -1 && sV[i] > -1) {
      double a = (Ic - (sI[i] - sV[i]));
      x += (a * (c->lambda[i] - l0));
      y += a;
    }
  lm = (fabs(y) > 1e-15) ? x / y : 0;
  C = (PMO_ZEEMAN * (l0 * l0) * c->geff);
  Blos = (1 / C) * ((lp - lm) / 2);
  Vlos = (PMO_VLIGHT / (l0)) * ((xv / yv) / 2);
  x = y = 0;
  for (i = begin; i < end - 1; i++)
    if (sQ[i] > -1 && sU[i] > -1 && sV[i] > -1) {
      double L = RFABS(RSQRT(sQ[i] * sQ[i] + sU[i] * sU[i]));
      double mm = fabs((4 * (c->lambda[i] - l0) * L));
      x = x + RFABS(sV[i]) * mm;
      y = y + RFABS(sV[i]) * RFABS(sV[i]);
    }
  y = y * fabs((3 * C * Blos));
  tan_gamma = fabs(sqrt(x / y));
  gamma_rad = atan(tan_gamma);
  gamma = gamma_rad * (180 / PMO_PI);
  if (initial_use) {
    if (gamma >= 85 && gamma <= 90) gamma_rad = 85 * (PMO_PI / 180);
    if (gamma > 90 && gamma <= 95) gamma_rad = 95 * (PMO_PI / 180);
  }
  if (Blos < 0) gamma = (180) - gamma;
  sum_u = sum_q = 0.0;
  for (i = 0; i < n; i++)
    if (sU[i] > -1 && sQ[i] > -1 && (fabs(sU[i]) > 0.0001 || fabs(sQ[i]) > 0.0001)) {
      sum_u += sU[i];
      sum_q += sQ[i];
    }
  tan2phi = sum_u / sum_q;
  phi = (atan(tan2phi) * 180 / PMO_PI) / 2;
  if (sum_u > 0 && sum_q > 0) phi = phi;
  else if (sum_u < 0 && sum_q > 0) phi = phi + 180;
  else if (sum_u < 0 && sum_q < 0) phi = phi + 90;
  else if (sum_u > 0 && sum_q < 0) phi = phi + 90;
  B_aux = fabs(Blos / cos(gamma_rad));
  if (Vlos < (-4)) Vlos = -4;
  if (Vlos > (4)) Vlos = 4;
  m[I_B] = (B_aux > 4000 ? 4000 : B_aux);
  m[I_VLOS] = Vlos;
  m[I_GM] = gamma;
  m[I_AZ] = phi;
  if (!initial_use) m[I_S0] = Blos;
}

void pmo_classical(const pmo_ctx *c, const float *spectro, double *m) { classical(c, spectro, m, 1); }

/* The classical-estimates-only mode of the drivers (NumberOfCycles < 0,
 * milos.c:399-520): forInitialUse = 0, no NaN fixes, no lm_mils. */
void pmo_classical_only(const pmo_ctx *c, const float *spectro, double *m) { classical(c, spectro, m, 0); }

/* ------------------------------------------------------------------ */
/* Levenberg-Marquardt driver: lm_mils, milosUtils.c:466-635.          */
/* ------------------------------------------------------------------ */
static int lm(pmo_ctx *c, const float *obs, double *model, float *chisqrf, const real *slight, double toplim,
              int miter, const real *w, const int *fix, real sigma, real ilambda, int *iter, real ah,
              int logclambda, int *accepted, int *why) {
  const int n = c->nl, K = c->K;
  const real better = 5.0, worse = 10.0;
  real factor = 1.0, flambda, chi, ochi, chi0;
  real beta[11], alpha[11 * 11];
  double covar[11 * 11], delta[11], trial[11];
  int i, ghosts = 0, nfree, stop = 0;
  *accepted = 0;
  *why = 2; /* the iteration cap, unless a stopping test ends the loop */
  for (i = 0; i < 4 * n; i++) {
    if (obs[i] <= -1) { c->vsigma[i] = (real)PMO_GHOST_SIGMA; ghosts++; }
    else c->vsigma[i] = sigma;
  }
  nfree = (4 * n - K) - ghosts;
  if (nfree == 0) return -1; /* 'NOT ENOUGH POINTS'; *iter is left as passed in */
  *iter = 0;
  flambda = ilambda;

  if (synthesis(c, model, ah, slight) != 0) return -3;
  response_functions(c, model, ah, slight, c->spectra_slight, fix);
  zero_fixed_rfs(c, fix);
  normal_equations(c, w, c->vsigma, obs, beta, alpha);
  for (i = 0; i < K * K; i++) covar[i] = alpha[i];
  ochi = chisq(c, obs, w, c->vsigma, (real)nfree);
  chi0 = ochi;
  for (i = 0; i < 11; i++) trial[i] = model[i];
  do {
    for (i = 0; i < K; i++) covar[i * (K + 1)] = alpha[i * (K + 1)] * (1.0 + flambda);
    svd_solve(K, covar, beta, delta);
    apply_delta(model, delta, fix, K, trial);
    clamp_model(trial);
    if (synthesis(c, trial, ah, slight) != 0) return -3;
    chi = chisq(c, obs, w, c->vsigma, (real)nfree);
    if ((RFABS((ochi - chi) * 100 / chi) < toplim) || (chi < 0.0001)) {
      stop = 1;
      *why = 0;
    }
    if (chi - ochi < 0.) {
      flambda = flambda / (better * factor);
      for (i = 0; i < 11; i++) model[i] = trial[i];
      response_functions(c, model, ah, slight, c->spectra, fix);
      zero_fixed_rfs(c, fix);
      normal_equations(c, w, c->vsigma, obs, beta, alpha);
      for (i = 0; i < K * K; i++) covar[i] = alpha[i];
      ochi = chi;
      (*accepted)++;
    } else {
      for (i = 0; i < K * K; i++) covar[i] = alpha[i];
      flambda = flambda * worse * factor;
    }
    if ((flambda > 1e+7) || (flambda < 1e-25)) {
      if (!stop) *why = 1;
      stop = 1;
    }
    (*iter)++;
    if (logclambda) factor = (real)(log10f((float)chi) / log10f((float)chi0));
  } while (*iter < miter && !stop);
  *chisqrf = (float)ochi;
  return 1;
}

static real *stage_slight(pmo_ctx *c, const double *slight) {
  int i;
  if (!slight) return NULL;
  for (i = 0; i < 4 * c->nl; i++) c->slight[i] = (real)slight[i];
  return c->slight;
}

int pmo_synth(pmo_ctx *c, const double *model, const double *slight, double mu, const int *fix,
              double *spectra_out, double *d_spectra_out) {
  int i, fx[11];
  real *sl = stage_slight(c, slight);
  for (i = 0; i < 11; i++) fx[i] = fix ? fix[i] : 1;
  if (synthesis(c, model, (real)mu, sl) != 0) return -3;
  if (spectra_out)
    for (i = 0; i < 4 * c->nl; i++) spectra_out[i] = c->spectra[i];
  if (d_spectra_out) {
    response_functions(c, model, (real)mu, sl, c->spectra_slight, fx);
    for (i = 0; i < 4 * c->nl * c->K; i++) d_spectra_out[i] = c->d_spectra[i];
  }
  return 0;
}

int pmo_invert_pixel(pmo_ctx *c, const float *spectro, const double *guess, const double *slight,
                     int use_classical, int miter, const double *w, double noise, double ilambda,
                     int logclambda, double toplim, double mu, const int *fix, double *model_out,
                     float *chisq_out, int *iters, double *spectra_out, pmo_stats *stats) {
  double m[11];
  real ww[4];
  int i, it = -1, acc = 0, why = 2, rc;
  float chi = 0.0f;
  real *sl = stage_slight(c, slight);
  for (i = 0; i < 4; i++) ww[i] = (real)w[i];
  for (i = 0; i < 11; i++) m[i] = guess[i];
  if (use_classical) {
    /* milos.c:975-983 */
    pmo_classical(c, spectro, m);
    if (isnan(m[I_B])) m[I_B] = 1;
    if (isnan(m[I_VLOS])) m[I_VLOS] = 1e-3;
    if (isnan(m[I_GM])) m[I_GM] = 1;
    if (isnan(m[I_AZ])) m[I_AZ] = 1;
  }
  rc = lm(c, spectro, m, &chi, sl, toplim, miter, ww, fix, (real)noise, (real)ilambda, &it, (real)mu, logclambda,
          &acc, &why);
  for (i = 0; i < 11; i++) model_out[i] = m[i];
  if (chisq_out) *chisq_out = chi;
  if (iters) *iters = it;
  if (spectra_out)
    for (i = 0; i < 4 * c->nl; i++) spectra_out[i] = c->spectra[i];
  if (stats) { stats->iterations = it; stats->accepted = acc; stats->status = rc == 1 ? why : rc; }
  return rc;
}

int pmo_invert_batch(pmo_ctx *c, int npix, const float *spectro, const double *guess, const double *slight,
                     int slight_per_pixel, int use_classical, int miter, const double *w, double noise,
                     double ilambda, int logclambda, double toplim, double mu, const int *fix,
                     double *models_out, float *chisq_out, int *iters_out, float *spectra_out,
                     int *accepted_out, int *status_out) {
  const size_t n4 = (size_t)4 * c->nl;
  double *sp = spectra_out ? (double *)malloc(sizeof(double) * n4) : NULL;
  int p;
  size_t i;
  for (p = 0; p < npix; p++) {
    const double *slp = slight ? (slight_per_pixel ? slight + (size_t)p * n4 : slight) : NULL;
    pmo_stats st;
    pmo_invert_pixel(c, spectro + (size_t)p * n4, guess, slp, use_classical, miter, w, noise, ilambda, logclambda,
                     toplim, mu, fix, models_out + (size_t)p * 11, chisq_out + p, iters_out + p, sp, &st);
    if (accepted_out) accepted_out[p] = st.accepted;
    if (status_out) status_out[p] = st.status;
    if (sp)
      for (i = 0; i < n4; i++) spectra_out[(size_t)p * n4 + i] = (float)sp[i];
  }
  free(sp);
  return 0;
}
