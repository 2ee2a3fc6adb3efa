// pm_host.cpp -- host side of libpmilos_b200.so: the C ABI of include/pmilos.h.
//
// Responsibilities: per-run precompute that the reference does on the host
// (Zeeman pattern, PSF taps), validation of the control settings, the context
// (parameter block, device staging buffers, counters), and the batched entry
// points that replace the reference's per-pixel loops.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "pm_params.h"

namespace {

thread_local char g_last_error[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof g_last_error, fmt, ap);
  va_end(ap);
  return code;
}

int cuda_fail(cudaError_t e, const char* what, int code = PM_EIO) {
  return fail(code, "%s: %s", what, cudaGetErrorString(e));
}

#define PM_CUDA(call, what)                       \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

// A start/stop event pair that every return path of its owner releases.
struct TimingEvents {
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  cudaError_t create() {
    cudaError_t e = cudaEventCreate(&t0);
    return e != cudaSuccess ? e : cudaEventCreate(&t1);
  }
  ~TimingEvents() {
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
  }
};

// Device buffer that grows on demand.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return PM_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) return fail(PM_ENOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    cap = bytes;
    return PM_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

}  // namespace

// Pinned host words the streamed calls copy from and read back into.
struct HostCtl {
  unsigned long long one;                    // 1: the value of PmStreamQ::closed
  PmJob job;
  PmStreamQ qinit;                           // queue state before a fully published launch
  PmStreamQ qread;                           // queue state after the kernel (counters, err)
  unsigned long long piece_avail[PM_STAGING_MAX];  // tickets published once piece i of a streamed call is in
  unsigned long long wide_ctr[2][PMC_COUNT];  // counters of the two buffer sets of a wide-grid call
};

// A captured CUDA graph of a whole small host-buffer call (uploads from pinned
// staging, job and queue, kernel, downloads into pinned staging) and what it
// was captured for: a replay is valid while all of these are unchanged.
struct SmallGraph {
  cudaGraphExec_t exec = nullptr;
  int64_t npix = -1;
  int slight_mode = -1;
  bool spectra = false, status = false;
  pm_tuning tuning{};
  void* dev[8] = {};
  std::vector<unsigned char> params;
};
constexpr int kGraphCache = 4;
constexpr size_t kProfMax = sizeof(float) * 4 * 32;  // one pixel's profiles, one-warp grids

// Pinned staging of the graph path, PM_GRAPH_MAX_PIXELS pixels of each array.
struct SmallStage {
  float spectro[PM_GRAPH_MAX_PIXELS * 4 * 32];
  float slight[PM_GRAPH_MAX_PIXELS * 4 * 32];
  float spectra[PM_GRAPH_MAX_PIXELS * 4 * 32];
  pm_model models[PM_GRAPH_MAX_PIXELS];
  float chisq[PM_GRAPH_MAX_PIXELS];
  int iters[PM_GRAPH_MAX_PIXELS];
  int status[PM_GRAPH_MAX_PIXELS];
};

struct pm_ctx {
  PmParams P;
  int precision = PM_PREC_FP32;
  pm_tuning tuning{2, 8, 16, 1};  // lock-step blocks of 16 warps (FP32 one-warp grids), fed in up to 8 pieces
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  // device staging of a host-buffer call (8 GiB; PMILOS_RESIDENT_MB at context
  // creation overrides it): larger cubes go in chunks
  size_t resident_bytes = size_t(8) << 30;
  DevBuf spectro, slight, models, chisq, iters, spectra, status, rf, ctr, lambda;
  // streamed host-buffer calls: kernel and copy streams, the ticket queue, one job
  cudaStream_t s_kern = nullptr, s_copy = nullptr;
  cudaEvent_t ev_start = nullptr, ev_q = nullptr, ev_done = nullptr, t0 = nullptr, t1 = nullptr, k0 = nullptr,
              k1 = nullptr;
  cudaEvent_t ev_piece[PM_STAGING_MAX] = {};  // a piece of a pipelined call is on the device
  DevBuf q, jobs;
  HostCtl* hc = nullptr;
  PmGridSet* gs = nullptr;  // kernel parameters of the streamed kernel (the context's one grid)
  SmallGraph graphs[kGraphCache];
  int graph_next = 0;
  SmallStage* stage = nullptr;  // pinned
  pm_stats stats{};
};

// ---------------------------------------------------------------------------
// Host precompute
// ---------------------------------------------------------------------------

// Zeeman pattern of an LS-coupled transition (Cuanten, create_cuantic.c:60-294):
// Lande factors of both levels, then for every pair of magnetic sublevels the
// component strength (by Delta J and Delta M) and splitting g1 M1 - g2 M2;
// strengths normalised per group.
extern "C" int pm_line_from_quantum(double lambda0, double sl, double ll, double jl, double su, double lu,
                                    double ju, pm_line* out) {
  if (!out) return fail(PM_EINVAL, "pm_line_from_quantum: out is NULL");
  if (!(lambda0 > 0) || jl < 0 || ju < 0 || std::fabs(ju - jl) > 1)
    return fail(PM_EINVAL, "pm_line_from_quantum: invalid line (lambda0=%g, jl=%g, ju=%g)", lambda0, jl, ju);
  std::memset(out, 0, sizeof *out);
  const double g1 = (jl != 0) ? (3.0 * jl * (jl + 1) + sl * (sl + 1) - ll * (ll + 1)) / (2 * jl * (jl + 1)) : 0;
  const double g2 =
      (ju != 0) ? (3.0 * ju * (ju + 1.0) + su * (su + 1.0) - lu * (lu + 1.0)) / (2.0 * ju * (ju + 1.0)) : 0;
  const double geff = (g1 + g2) / 2 + (g1 - g2) * (jl * (jl + 1.) - ju * (ju + 1.)) / 4;
  const int nlo = int(2 * jl + 1), nup = int(2 * ju + 1);
  const int jj = int(ju - jl);
  const int n_pi = int(2 * std::min(jl, ju) + 1), n_sig = int(jl + ju);
  if (n_pi > PM_ZEEMAN_MAX || n_sig > PM_ZEEMAN_MAX || n_sig < 1)
    return fail(PM_ERANGE, "pm_line_from_quantum: %d pi / %d sigma components exceed %d", n_pi, n_sig,
                PM_ZEEMAN_MAX);
  int ip = 0, ib = 0, ir = 0;
  for (int a = 0; a < nlo; ++a) {
    const int m1 = a - int(jl);
    for (int b = 0; b < nup; ++b) {
      const int m2 = b - int(ju);
      const int dm = m2 - m1;
      const double split = g1 * m1 - g2 * m2;
      if (dm == 0) {
        out->wep[ip] = (jj == -1) ? jl * jl - m1 * m1 : (jj == 0) ? double(m1 * m1) : (jl + 1) * (jl + 1) - m1 * m1;
        out->nup[ip++] = split;
      } else if (dm == 1) {
        out->web[ib] = (jj == -1)  ? (jl - m1) * (jl - m1 - 1) / 4
                       : (jj == 0) ? (jl - m1) * (jl + m1 + 1) / 4
                                   : (jl + m1 + 1) * (jl + m1 + 2) / 4;
        out->nub[ib++] = split;
      } else if (dm == -1) {
        out->wer[ir] = (jj == -1)  ? (jl + m1) * (jl + m1 - 1) / 4
                       : (jj == 0) ? (jl + m1) * (jl - m1 + 1) / 4
                                   : (jl - m1 + 1) * (jl - m1 + 2) / 4;
        out->nur[ir++] = split;
      }
    }
  }
  if (ip != n_pi || ib != n_sig || ir != n_sig) return fail(PM_EINVAL, "pm_line_from_quantum: inconsistent pattern");
  double s;
  s = 0; for (int k = 0; k < n_pi; ++k) s += out->wep[k];
  for (int k = 0; k < n_pi; ++k) out->wep[k] /= s;
  s = 0; for (int k = 0; k < n_sig; ++k) s += out->web[k];
  for (int k = 0; k < n_sig; ++k) out->web[k] /= s;
  s = 0; for (int k = 0; k < n_sig; ++k) s += out->wer[k];
  for (int k = 0; k < n_sig; ++k) out->wer[k] /= s;
  out->lambda0 = lambda0;
  out->n_pi = n_pi;
  out->n_sig = n_sig;
  out->gl = g1;
  out->gu = g2;
  out->geff = geff;
  out->fo = 1.0;
  return PM_OK;
}

// fgauss_WL (fgauss.c:79-154): sigma = FWHM * 0.42466090 / 1000 [A], centred on
// the grid's middle sample lambda[nl/2], sampled at lambda[0] + i * step with
// step = lambda[1] - lambda[0], normalised to unit sum.
extern "C" int pm_psf_gaussian(double fwhm_ma, int nlambda, const double* lambda, double* taps_out) {
  if (nlambda < 2 || !lambda || !taps_out || !(fwhm_ma > 0))
    return fail(PM_EINVAL, "pm_psf_gaussian: bad arguments");
  const double sigma = fwhm_ma * 0.42466090 / 1000.0;
  const double step = lambda[1] - lambda[0], first = lambda[0], central = lambda[nlambda / 2];
  double cte = 0;
  for (int i = 0; i < nlambda; ++i) {
    const double x = first + i * step;
    const double aux = (x - central) / sigma;
    const double term = (aux * aux) / 2;
    taps_out[i] = term < 1e30 ? std::exp(-term) : 0.0;
    cte += taps_out[i];
  }
  for (int i = 0; i < nlambda; ++i) taps_out[i] /= cte;
  return PM_OK;
}

// PSF from a tabulated file (readPSFFile + milos.c:302-344 + interpolationLinearPSF
// milosUtils.c:684-738).  The grid must lie inside the table (integer-truncated
// comparison); if the grid's zero offset is not its middle sample the table is
// shifted so that it is (quirk kept: the zero search stops at the first
// non-leading match); samples are linearly interpolated and normalised.
extern "C" int pm_psf_interpolate(int nsamples, const double* dl, const double* psf, int nlambda,
                                  const double* offs, double* taps_out) {
  if (nsamples < 2 || nlambda < 2 || !dl || !psf || !offs || !taps_out)
    return fail(PM_EINVAL, "pm_psf_interpolate: bad arguments");
  if (std::trunc(offs[0]) < std::trunc(dl[0]) || std::trunc(offs[nlambda - 1]) > std::trunc(dl[nsamples - 1]))
    return fail(PM_EINVAL, "pm_psf_interpolate: PSF table [%g,%g] mA does not cover the grid [%g,%g] mA", dl[0],
                dl[nsamples - 1], offs[0], offs[nlambda - 1]);
  int posWL = 0;
  for (int i = 0; i < nlambda && !posWL; ++i)
    if (std::fabs(std::trunc(offs[i])) == 0) posWL = i;
  double offset = 0;
  const double step = (offs[1] - offs[0]) / 1000.0;
  if (posWL != nlambda / 2) offset = ((nlambda / 2 - posWL) * step) * 1000;
  auto interp = [&](double x, double* y) -> bool {
    if (!(x >= dl[0] && x <= dl[nsamples - 1])) return false;
    int lo = 0, hi = nsamples - 1;
    while (hi > lo + 1) {
      const int mid = (lo + hi) / 2;
      if (dl[mid] > x) hi = mid; else lo = mid;
    }
    const double dx = dl[lo + 1] - dl[lo];
    *y = dx > 0 ? psf[lo] + (x - dl[lo]) / dx * (psf[lo + 1] - psf[lo]) : 0.0;
    return true;
  };
  for (int i = 0; i < nlambda; ++i) {
    taps_out[i] = 0.0;
    const double x = offs[i] - offset;
    const double lower = (offset >= 0) ? dl[0] : dl[std::min(nlambda, nsamples) - 1];
    double y;
    if (x >= lower && interp(x, &y)) taps_out[i] = y;
  }
  double cte = 0;
  for (int i = 0; i < nlambda; ++i) cte += taps_out[i];
  for (int i = 0; i < nlambda; ++i) taps_out[i] /= cte;
  return PM_OK;
}

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
namespace {

int fill_params(const pm_line* L, const pm_config* c, PmParams& P) {
  std::memset(&P, 0, sizeof P);
  if (c->nlambda < 2 || c->nlambda > PMK_NL)
    return fail(PM_ERANGE, "nlambda=%d: this build handles 2..%d wavelengths", c->nlambda, PMK_NL);
  if (!c->lambda) return fail(PM_EINVAL, "lambda grid is NULL");
  if (c->nterms < 9 || c->nterms > 11) return fail(PM_ENOTSUP, "nterms=%d: supported are 9, 10 and 11", c->nterms);
  {
    // NTERMS = 11 - !fix[10] - (mac == 0 && !fix[9]) (milos.c:152-157); the
    // guess's v_mac settles the last term when the guess is known (pmh_check_guess)
    const int hi = 11 - (c->fix[10] ? 0 : 1);
    const int lo = hi - (c->fix[9] ? 0 : 1);
    if (c->nterms < lo || c->nterms > hi)
      return fail(PM_EINVAL, "nterms=%d inconsistent with fix[9]=%d, fix[10]=%d (expected %d..%d)", c->nterms,
                  c->fix[9], c->fix[10], lo, hi);
  }
  if (!(c->noise > 0)) return fail(PM_EINVAL, "noise must be > 0");
  if (c->precision != PM_PREC_FP32 && c->precision != PM_PREC_FP64) return fail(PM_EINVAL, "precision");
  if (L->n_pi < 1 || L->n_sig < 1 || L->n_pi > PM_ZEEMAN_MAX || L->n_sig > PM_ZEEMAN_MAX)
    return fail(PM_EINVAL, "Zeeman pattern with %d pi and %d sigma components (1..%d per group)", L->n_pi,
                L->n_sig, PM_ZEEMAN_MAX);
  P.nl = c->nlambda;
  P.half = c->nlambda / 2;
  P.K = c->nterms;
  P.miter = c->miter;  // < 0: classical estimates alone (NumberOfCycles < 0, milos.c:399-520)
  P.nfree_base = 4 * c->nlambda - c->nterms;
  P.logclambda = c->logclambda;
  P.classical = c->classical_estimates;
  P.has_psf = c->psf != nullptr;
  int solver = c->solver;
  if (solver == PM_SOLVE_DEFAULT) solver = (c->precision == PM_PREC_FP64) ? PM_SOLVE_EIGEN : PM_SOLVE_CHOLESKY;
  if (solver != PM_SOLVE_EIGEN && solver != PM_SOLVE_CHOLESKY) return fail(PM_EINVAL, "solver=%d", c->solver);
  P.solver = solver;
  P.n_pi = L->n_pi;
  P.n_sig = L->n_sig;
  for (int i = 0; i < 11; ++i) P.fix[i] = c->fix[i] ? 1 : 0;
  // FijaACeroDerivadasNoNecesarias (milosUtils.c:199-227)
  for (int k = 0; k < P.K; ++k) {
    if (P.K == 10 && k == 9) P.zero_row[k] = (P.fix[9] == 0 && P.fix[10] == 0);
    else P.zero_row[k] = (P.fix[k] == 0);
  }
  // me_der.c:499-525: the filling-factor row is 10 with NTERMS 11, else 9 unless
  // v_mac is inverted; row 9 is v_mac's with NTERMS 11 or 10 and alpha fixed
  P.ff_row = (P.K == 11) ? 10 : ((P.K == 10 && !P.fix[9]) ? 9 : -1);
  P.mac_row = (P.K == 11 || (P.K == 10 && !P.fix[10])) ? 9 : -1;
  P.lambda0 = L->lambda0;
  for (int i = 0; i < P.nl; ++i) P.dl[i] = c->lambda[i] - L->lambda0;
  for (int k = 0; k < L->n_pi; ++k) { P.nu[0][k] = L->nup[k]; P.we[0][k] = L->wep[k]; }
  for (int k = 0; k < L->n_sig; ++k) {
    P.nu[1][k] = L->nub[k];
    P.we[1][k] = L->web[k];
    P.nu[2][k] = -L->nub[L->n_sig - 1 - k];  // mil_sinrf.c:164-166 mirrors the blue splitting
    P.we[2][k] = L->wer[k];
  }
  P.geff = L->geff;
  P.fo = L->fo;
  for (int s = 0; s < 4; ++s) P.w[s] = c->weight[s];
  P.noise = c->noise;
  P.ilambda = c->ilambda;
  P.toplim = c->toplim;
  P.mu = c->mu;
  P.G = P.nl <= 32 ? 1 : (P.nl <= 64 ? 2 : 4);
  if (c->psf) {
    double peak = 0;
    for (int j = 0; j < P.nl; ++j) {
      P.taps_d[j] = c->psf[j];
      P.taps_f[j] = float(c->psf[j]);
      peak = std::max(peak, std::fabs(c->psf[j]));
    }
    // Support of the kernel for the multi-warp correlations: taps below 1e-18 of
    // the peak change no output by more than 1e-18 of the largest input.
    P.tap_lo = 0;
    P.tap_hi = P.nl - 1;
    while (P.tap_lo < P.tap_hi && !(std::fabs(c->psf[P.tap_lo]) > 1e-18 * peak)) ++P.tap_lo;
    while (P.tap_hi > P.tap_lo && !(std::fabs(c->psf[P.tap_hi]) > 1e-18 * peak)) --P.tap_hi;
    // Stokes I is correlated as Ic - x (direct_convolution_ic): with zero padding
    // that is Ic (1 - W_k) + sum_j G_j x_{k+j-half}, W_k the in-grid tap sum.
    for (int k = 0; k < P.nl; ++k) {
      double w = 0;
      for (int j = P.tap_lo; j <= P.tap_hi; ++j) {
        const int m = k + j - P.half;
        if (m >= 0 && m < P.nl) w += c->psf[j];
      }
      P.omw_d[k] = 1.0 - w;
      P.omw_f[k] = float(1.0 - w);
    }
  }
  return PM_OK;
}

void set_guess(PmParams& P, const pm_model* g) {
  const double* v = reinterpret_cast<const double*>(g);
  for (int i = 0; i < 11; ++i) P.guess[i] = v[i];
}

// NTERMS = 11 - !fix[10] - (mac == 0 && !fix[9]) (milos.c:152-157), now that the
// guess's v_mac is known.
int check_guess(const PmParams& P, const pm_model* g) {
  const int expect = 11 - (P.fix[10] ? 0 : 1) - ((g->mac == 0.0 && !P.fix[9]) ? 1 : 0);
  if (expect != P.K)
    return fail(PM_EINVAL, "nterms=%d inconsistent with guess v_mac=%g, fix[9]=%d, fix[10]=%d (NTERMS would be %d)", P.K,
                g->mac, P.fix[9], P.fix[10], expect);
  return PM_OK;
}

int set_slight(PmParams& P, const float* slight, int mode, int mem) {
  P.slight_mode = mode;
  if (mode == PM_SLIGHT_NONE) return PM_OK;
  if (!slight) return fail(PM_EINVAL, "slight_mode=%d but slight is NULL", mode);
  if (P.K < 10) return fail(PM_EINVAL, "stray light requires nterms >= 10 (filling factor or v_mac inverted)");
  if (mode == PM_SLIGHT_SHARED) {
    std::vector<float> h(4 * P.nl);
    if (mem == PM_MEM_DEVICE) {
      cudaError_t e = cudaMemcpy(h.data(), slight, sizeof(float) * 4 * P.nl, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) return cuda_fail(e, "slight D2H");
    } else {
      std::memcpy(h.data(), slight, sizeof(float) * 4 * P.nl);
    }
    for (int i = 0; i < 4 * P.nl; ++i) {
      P.sl_f[i] = h[i];
    }
    return PM_OK;
  }
  if (mode == PM_SLIGHT_PER_PIXEL) return PM_OK;
  return fail(PM_EINVAL, "slight_mode=%d", mode);
}

}  // namespace

// Helpers shared with the other translation units of the library.
int pmh_fill_params(const pm_line* L, const pm_config* c, PmParams& P) { return fill_params(L, c, P); }
void pmh_set_guess(PmParams& P, const pm_model* g) { set_guess(P, g); }
int pmh_check_guess(const PmParams& P, const pm_model* g) { return check_guess(P, g); }
int pmh_fail(int code, const char* msg) { return fail(code, "%s", msg); }
int pmh_set_slight(PmParams& P, const float* slight, int mode) { return set_slight(P, slight, mode, PM_MEM_HOST); }

extern "C" int pm_ctx_create(const pm_line* line, const pm_config* cfg, void* stream, pm_ctx** out) {
  if (!line || !cfg || !out) return fail(PM_EINVAL, "pm_ctx_create: NULL argument");
  *out = nullptr;
  pm_ctx* c = new (std::nothrow) pm_ctx();
  if (!c) return fail(PM_ENOMEM, "pm_ctx_create: out of host memory");
  int rc = fill_params(line, cfg, c->P);
  if (rc != PM_OK) {
    delete c;
    return rc;
  }
  c->precision = cfg->precision;
  c->stream = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaGetDevice(&c->device);
  cudaDeviceProp prop;
  if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, c->device);
  if (e != cudaSuccess) {
    delete c;
    return fail(PM_ENODEV, "no CUDA device: %s", cudaGetErrorString(e));
  }
  if (prop.major != 10) {
    delete c;
    return fail(PM_ENODEV, "device %d is sm_%d%d; this library is built for sm_100a", c->device, prop.major,
                prop.minor);
  }
  c->num_sms = prop.multiProcessorCount;
  if (const char* v = std::getenv("PMILOS_VARIANT")) {
    const int var = std::atoi(v);
    if (var >= 0 && var <= 2) c->tuning.variant = var;
    if (c->tuning.variant != 2) c->tuning.warps_per_block = 4;
  }
  if (const char* v = std::getenv("PMILOS_RESIDENT_MB"))
    if (std::atoll(v) > 0) c->resident_bytes = size_t(std::atoll(v)) << 20;
  if (const char* v = std::getenv("PMILOS_STAGING")) c->tuning.staging_depth = std::atoi(v);
  rc = c->ctr.ensure(sizeof(unsigned long long) * PMC_COUNT);
  if (rc != PM_OK) {
    delete c;
    return rc;
  }
  *out = c;
  return PM_OK;
}

extern "C" int pm_ctx_destroy(pm_ctx* c) {
  if (!c) return PM_OK;
  PmDeviceGuard dg(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  else cudaDeviceSynchronize();
  if (c->s_kern) cudaStreamSynchronize(c->s_kern);
  if (c->s_copy) cudaStreamSynchronize(c->s_copy);
  for (DevBuf* b : {&c->spectro, &c->slight, &c->models, &c->chisq, &c->iters, &c->spectra, &c->status, &c->rf,
                    &c->ctr, &c->q, &c->jobs, &c->lambda})
    b->release();
  for (cudaEvent_t ev : {c->ev_start, c->ev_q, c->ev_done, c->t0, c->t1, c->k0, c->k1})
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : c->ev_piece)
    if (ev) cudaEventDestroy(ev);
  if (c->s_kern) cudaStreamDestroy(c->s_kern);
  if (c->s_copy) cudaStreamDestroy(c->s_copy);
  if (c->hc) cudaFreeHost(c->hc);
  if (c->stage) cudaFreeHost(c->stage);
  for (SmallGraph& g : c->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  delete c->gs;
  delete c;
  return PM_OK;
}

namespace {

// Resources of the streamed launches, created on first use.
int stream_resources(pm_ctx* c) {
  if (c->hc) return PM_OK;
  PM_CUDA(cudaStreamCreateWithFlags(&c->s_kern, cudaStreamNonBlocking), "stream create");
  PM_CUDA(cudaStreamCreateWithFlags(&c->s_copy, cudaStreamNonBlocking), "stream create");
  for (cudaEvent_t* ev : {&c->ev_start, &c->ev_q, &c->ev_done})
    PM_CUDA(cudaEventCreateWithFlags(ev, cudaEventDisableTiming), "event create");
  for (cudaEvent_t* ev : {&c->t0, &c->t1, &c->k0, &c->k1}) PM_CUDA(cudaEventCreate(ev), "event create");
  for (cudaEvent_t& ev : c->ev_piece) PM_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event create");
  int rc = c->q.ensure(sizeof(PmStreamQ));
  if (rc == PM_OK) rc = c->jobs.ensure(sizeof(PmJob));
  if (rc != PM_OK) return rc;
  c->gs = new (std::nothrow) PmGridSet();
  if (!c->gs) return fail(PM_ENOMEM, "out of host memory");
  void* h = nullptr;
  PM_CUDA(cudaHostAlloc(&h, sizeof(HostCtl), cudaHostAllocDefault), "cudaHostAlloc");
  std::memset(h, 0, sizeof(HostCtl));
  c->hc = static_cast<HostCtl*>(h);
  c->hc->one = 1;
  return PM_OK;
}

// The device address of host range [p, p + bytes) when the whole range is
// pinned, mapped memory (cudaHostAlloc, or cudaHostRegister with mapping), else
// nullptr: a kernel can then store results into it directly.
void* mapped_host_range(const void* p, size_t bytes) {
  if (!p || bytes == 0) return nullptr;
  cudaPointerAttributes a{}, b{};
  const char* last = static_cast<const char*>(p) + bytes - 1;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess || cudaPointerGetAttributes(&b, last) != cudaSuccess) {
    cudaGetLastError();  // not a pointer CUDA knows: pageable
    return nullptr;
  }
  if (a.type != cudaMemoryTypeHost || b.type != cudaMemoryTypeHost || !a.devicePointer || !b.devicePointer)
    return nullptr;
  if (static_cast<const char*>(b.devicePointer) - static_cast<const char*>(a.devicePointer) != ptrdiff_t(bytes - 1))
    return nullptr;
  return a.devicePointer;
}

// One resident chunk of a host-buffer inversion: one persistent launch fed while
// it runs.  The cube goes to the device in up to `staging_depth` copies on the
// copy stream, each twice the size of the one before (multiples of 32 pixels,
// so no 128-byte line of the cube spans two), so the first publication follows
// a copy of a few hundred pixels; after each copy the copy stream writes the
// running pixel count into the queue's avail word, which publishes that piece's
// tickets to the kernel already running on the kernel stream.  The kernel
// computes each pixel's classical estimates itself (a pre-pass launch could not
// find SM slots beside the persistent kernel).  Results go straight into the
// caller's buffers when those are pinned and mapped (each pixel's stores cross
// the bus as the pixel ends, nothing is left to copy after the kernel), else
// they come back in one copy after the kernel.
int run_streamed(pm_ctx* c, int64_t n, const float* spectro, const float* slight, int slight_mode,
                 pm_model* models_out, float* chisq_out, int* iters_out, float* best_fit_out, int* status_out,
                 float* kernel_ms, float* total_ms) {
  int rc = stream_resources(c);
  if (rc != PM_OK) return rc;
  const int nl = c->P.nl;
  const size_t prof = sizeof(float) * 4 * nl;
  HostCtl* hc = c->hc;
  PmStreamQ* q = static_cast<PmStreamQ*>(c->q.p);
  c->gs->ngrids = 1;
  c->gs->g[0] = c->P;
  PmStreamIO sio{};
  sio.q = q;
  sio.jobs = static_cast<const PmJob*>(c->jobs.p);
  sio.jobs_cap = 1;
  sio.first_job = 0;
  sio.wait_limit_ns = 20000000000LL;

  // piece i holds first << i pixels (the last one the rest): at most `depth` pieces
  const int depth = std::max(1, std::min(c->tuning.staging_depth, PM_STAGING_MAX));
  const double units = std::ldexp(1.0, std::min(depth, 40)) - 1.0;
  const int64_t first = std::max<int64_t>(32, (int64_t(std::ceil(double(n) / units)) + 31) / 32 * 32);

  // outputs the kernel can store into directly
  double* models_dev = static_cast<double*>(mapped_host_range(models_out, sizeof(pm_model) * n));
  float* chisq_dev = static_cast<float*>(mapped_host_range(chisq_out, sizeof(float) * n));
  int* iters_dev = static_cast<int*>(mapped_host_range(iters_out, sizeof(int) * n));
  int* status_dev = status_out ? static_cast<int*>(mapped_host_range(status_out, sizeof(int) * n)) : nullptr;
  float* spectra_dev = best_fit_out ? static_cast<float*>(mapped_host_range(best_fit_out, prof * n)) : nullptr;

  PmJob& job = hc->job;
  std::memset(&job, 0, sizeof job);
  job.npix = n;
  job.spectro = static_cast<const float*>(c->spectro.p);
  job.slight = slight_mode == PM_SLIGHT_PER_PIXEL ? static_cast<const float*>(c->slight.p) : nullptr;
  job.models = models_dev ? models_dev : static_cast<double*>(c->models.p);
  job.chisq = chisq_dev ? chisq_dev : static_cast<float*>(c->chisq.p);
  job.iters = iters_dev ? iters_dev : static_cast<int*>(c->iters.p);
  job.status = status_out ? (status_dev ? status_dev : static_cast<int*>(c->status.p)) : nullptr;
  job.spectra = best_fit_out ? (spectra_dev ? spectra_dev : static_cast<float*>(c->spectra.p)) : nullptr;
  job.model_in = nullptr;  // classical estimates in the kernel
  std::memset(&hc->qinit, 0, sizeof hc->qinit);  // nothing published, queue open

  // order after the caller's earlier work on its stream
  PM_CUDA(cudaEventRecord(c->ev_start, c->stream), "event");
  PM_CUDA(cudaStreamWaitEvent(c->s_copy, c->ev_start, 0), "wait");
  PM_CUDA(cudaStreamWaitEvent(c->s_kern, c->ev_start, 0), "wait");
  PM_CUDA(cudaEventRecord(c->t0, c->s_kern), "event");
  PM_CUDA(cudaMemcpyAsync(c->jobs.p, &job, sizeof job, cudaMemcpyHostToDevice, c->s_kern), "job H2D");
  PM_CUDA(cudaMemcpyAsync(q, &hc->qinit, sizeof(PmStreamQ), cudaMemcpyHostToDevice, c->s_kern), "queue H2D");
  PM_CUDA(cudaEventRecord(c->ev_q, c->s_kern), "event");  // the queue is reset: publications may follow
  PM_CUDA(cudaEventRecord(c->k0, c->s_kern), "event");
  rc = pmk_invert_stream(*c->gs, sio, c->precision, c->tuning.variant, c->tuning.warps_per_block, false, c->s_kern,
                         c->num_sms, nullptr);
  if (rc != PM_OK) {
    // the kernel did not start: nothing waits for the publications below
    cudaStreamSynchronize(c->s_kern);
    return fail(rc, "%s", pmk_last_cuda_error());
  }
  PM_CUDA(cudaEventRecord(c->k1, c->s_kern), "event");
  int64_t p0 = 0;
  for (int i = 0; p0 < n; ++i) {
    const int64_t m = i + 1 < PM_STAGING_MAX ? std::min(first << std::min(i, 40), n - p0) : n - p0;
    PM_CUDA(cudaMemcpyAsync(static_cast<char*>(c->spectro.p) + prof * p0, spectro + p0 * 4 * nl, prof * m,
                            cudaMemcpyHostToDevice, c->s_copy),
            "spectro H2D");
    if (slight_mode == PM_SLIGHT_PER_PIXEL)
      PM_CUDA(cudaMemcpyAsync(static_cast<char*>(c->slight.p) + prof * p0, slight + p0 * 4 * nl, prof * m,
                              cudaMemcpyHostToDevice, c->s_copy),
              "slight H2D");
    if (i == 0) PM_CUDA(cudaStreamWaitEvent(c->s_copy, c->ev_q, 0), "wait");
    hc->piece_avail[i] = (unsigned long long)(p0 + m);
    PM_CUDA(cudaMemcpyAsync(&q->avail, &hc->piece_avail[i], sizeof(unsigned long long), cudaMemcpyHostToDevice,
                            c->s_copy),
            "publish");
    p0 += m;
  }
  // closed after the last publication: warps holding tickets beyond n exit
  PM_CUDA(cudaMemcpyAsync(&q->closed, &hc->one, sizeof(unsigned long long), cudaMemcpyHostToDevice, c->s_copy),
          "close");
  if (!models_dev)
    PM_CUDA(cudaMemcpyAsync(models_out, job.models, sizeof(pm_model) * n, cudaMemcpyDeviceToHost, c->s_kern),
            "models D2H");
  if (!chisq_dev)
    PM_CUDA(cudaMemcpyAsync(chisq_out, job.chisq, sizeof(float) * n, cudaMemcpyDeviceToHost, c->s_kern), "chisq D2H");
  if (!iters_dev)
    PM_CUDA(cudaMemcpyAsync(iters_out, job.iters, sizeof(int) * n, cudaMemcpyDeviceToHost, c->s_kern), "iters D2H");
  if (best_fit_out && !spectra_dev)
    PM_CUDA(cudaMemcpyAsync(best_fit_out, job.spectra, prof * n, cudaMemcpyDeviceToHost, c->s_kern), "best fit D2H");
  if (status_out && !status_dev)
    PM_CUDA(cudaMemcpyAsync(status_out, job.status, sizeof(int) * n, cudaMemcpyDeviceToHost, c->s_kern),
            "status D2H");
  PM_CUDA(cudaMemcpyAsync(&hc->qread, q, sizeof(PmStreamQ), cudaMemcpyDeviceToHost, c->s_kern), "queue D2H");
  PM_CUDA(cudaEventRecord(c->t1, c->s_kern), "event");
  PM_CUDA(cudaEventRecord(c->ev_done, c->s_kern), "event");
  PM_CUDA(cudaStreamWaitEvent(c->stream, c->ev_done, 0), "wait");
  // the copy stream's last publication is done once the kernel has ended
  PM_CUDA(cudaStreamWaitEvent(c->s_copy, c->ev_done, 0), "wait");
  PM_CUDA(cudaEventSynchronize(c->t1), "streamed inversion");
  const PmStreamQ& r = hc->qread;
  if (r.err || r.next < (unsigned long long)n)
    return fail(PM_EIO, "streamed inversion: queue error %llu, %llu of %lld pixels handed out", r.err, r.next,
                (long long)n);
  c->stats.iterations += int64_t(r.ctr[PMC_ITERS]);
  c->stats.accepted += int64_t(r.ctr[PMC_ACCEPTED]);
  c->stats.eigen_fallbacks += int64_t(r.ctr[PMC_FALLBACK]);
  cudaEventElapsedTime(kernel_ms, c->k0, c->k1);
  cudaEventElapsedTime(total_ms, c->t0, c->t1);
  c->stats.pixels += n;
  return PM_OK;
}

// A host-buffer call on a grid wider than one warp, in chunks through two
// device buffer sets: the copy stream brings chunk k + 1 into one set while the
// kernel stream inverts chunk k in the other (classical pre-pass + LM kernel),
// and chunk k's results leave on the copy stream once its kernel is done.  A set
// is refilled only after its results are out (stream order on the copy
// stream), and a kernel starts only after its chunk is in (event).  Each set's
// work counter is reset per launch; its statistics counters add up over the
// set's launches and are read once at the end.
int run_wide_pipelined(pm_ctx* c, int64_t npix, int64_t chunk, const float* spectro, const float* slight,
                       int slight_mode, pm_model* models_out, float* chisq_out, int* iters_out, float* best_fit_out,
                       int* status_out, float* kernel_ms) {
  int rc = stream_resources(c);
  if (rc != PM_OK) return rc;
  const int nl = c->P.nl;
  const size_t prof = sizeof(float) * 4 * nl;
  const bool per_pixel = slight_mode == PM_SLIGHT_PER_PIXEL;
  if ((rc = c->ctr.ensure(2 * sizeof(unsigned long long) * PMC_COUNT)) != PM_OK) return rc;
  unsigned long long* ctr = static_cast<unsigned long long*>(c->ctr.p);
  HostCtl* hc = c->hc;
  cudaEvent_t ev_in[2] = {c->ev_piece[0], c->ev_piece[1]}, ev_k[2] = {c->ev_piece[2], c->ev_piece[3]};
  PM_CUDA(cudaEventRecord(c->ev_start, c->stream), "event");
  PM_CUDA(cudaStreamWaitEvent(c->s_copy, c->ev_start, 0), "wait");
  PM_CUDA(cudaStreamWaitEvent(c->s_kern, c->ev_start, 0), "wait");
  PM_CUDA(cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned long long) * PMC_COUNT, c->s_kern), "counter reset");
  const int64_t nchunks = (npix + chunk - 1) / chunk;
  // chunk k's inputs into set k & 1, then the event its kernel waits for
  auto copy_in = [&](int64_t k) -> int {
    const int b = int(k & 1);
    const int64_t p0 = k * chunk, n = std::min(chunk, npix - p0);
    PM_CUDA(cudaMemcpyAsync(static_cast<char*>(c->spectro.p) + prof * chunk * b, spectro + p0 * 4 * nl, prof * n,
                            cudaMemcpyHostToDevice, c->s_copy),
            "spectro H2D");
    if (per_pixel)
      PM_CUDA(cudaMemcpyAsync(static_cast<char*>(c->slight.p) + prof * chunk * b, slight + p0 * 4 * nl, prof * n,
                              cudaMemcpyHostToDevice, c->s_copy),
              "slight H2D");
    PM_CUDA(cudaEventRecord(ev_in[b], c->s_copy), "event");
    return PM_OK;
  };
  if ((rc = copy_in(0)) != PM_OK) return rc;
  for (int64_t k = 0; k < nchunks; ++k) {
    const int b = int(k & 1);
    const int64_t p0 = k * chunk, n = std::min(chunk, npix - p0);
    char* sp = static_cast<char*>(c->spectro.p) + prof * chunk * b;
    char* sl = per_pixel ? static_cast<char*>(c->slight.p) + prof * chunk * b : nullptr;
    PmIO io{};
    io.npix = n;
    io.spectro = reinterpret_cast<const float*>(sp);
    io.slight = reinterpret_cast<const float*>(sl);
    io.models_out = static_cast<double*>(c->models.p) + 11 * chunk * b;
    io.chisq_out = static_cast<float*>(c->chisq.p) + chunk * b;
    io.iters_out = static_cast<int*>(c->iters.p) + chunk * b;
    io.spectra_out = best_fit_out ? reinterpret_cast<float*>(static_cast<char*>(c->spectra.p) + prof * chunk * b)
                                  : nullptr;
    io.status_out = status_out ? static_cast<int*>(c->status.p) + chunk * b : nullptr;
    io.ctr = ctr + PMC_COUNT * b;
    PM_CUDA(cudaStreamWaitEvent(c->s_kern, ev_in[b], 0), "wait");
    PM_CUDA(cudaMemsetAsync(io.ctr + PMC_NEXT, 0, sizeof(unsigned long long), c->s_kern), "work counter reset");
    if (k == 0) PM_CUDA(cudaEventRecord(c->k0, c->s_kern), "event");
    rc = pmk_invert(c->P, io, c->precision, c->s_kern, c->num_sms, nullptr);
    if (rc != PM_OK) return fail(rc, "%s", pmk_last_cuda_error());
    if (k == nchunks - 1) PM_CUDA(cudaEventRecord(c->k1, c->s_kern), "event");
    PM_CUDA(cudaEventRecord(ev_k[b], c->s_kern), "event");
    // the next chunk goes in while this one is inverted: its copy is queued
    // before this chunk's results, which wait for this kernel; its set's previous
    // results (chunk k - 1) were queued before it
    if (k + 1 < nchunks && (rc = copy_in(k + 1)) != PM_OK) return rc;
    PM_CUDA(cudaStreamWaitEvent(c->s_copy, ev_k[b], 0), "wait");
    PM_CUDA(cudaMemcpyAsync(models_out + p0, io.models_out, sizeof(pm_model) * n, cudaMemcpyDeviceToHost, c->s_copy),
            "models D2H");
    PM_CUDA(cudaMemcpyAsync(chisq_out + p0, io.chisq_out, sizeof(float) * n, cudaMemcpyDeviceToHost, c->s_copy),
            "chisq D2H");
    PM_CUDA(cudaMemcpyAsync(iters_out + p0, io.iters_out, sizeof(int) * n, cudaMemcpyDeviceToHost, c->s_copy),
            "iters D2H");
    if (best_fit_out)
      PM_CUDA(cudaMemcpyAsync(best_fit_out + p0 * 4 * nl, io.spectra_out, prof * n, cudaMemcpyDeviceToHost, c->s_copy),
              "best fit D2H");
    if (status_out)
      PM_CUDA(cudaMemcpyAsync(status_out + p0, io.status_out, sizeof(int) * n, cudaMemcpyDeviceToHost, c->s_copy),
              "status D2H");
  }
  PM_CUDA(cudaStreamWaitEvent(c->s_copy, c->k1, 0), "wait");
  PM_CUDA(cudaMemcpyAsync(hc->wide_ctr, ctr, sizeof hc->wide_ctr, cudaMemcpyDeviceToHost, c->s_copy), "counter D2H");
  PM_CUDA(cudaEventRecord(c->ev_done, c->s_copy), "event");
  PM_CUDA(cudaStreamWaitEvent(c->stream, c->ev_done, 0), "wait");
  PM_CUDA(cudaEventSynchronize(c->ev_done), "wide inversion");
  for (int b = 0; b < 2; ++b) {
    c->stats.iterations += int64_t(hc->wide_ctr[b][PMC_ITERS]);
    c->stats.accepted += int64_t(hc->wide_ctr[b][PMC_ACCEPTED]);
    c->stats.eigen_fallbacks += int64_t(hc->wide_ctr[b][PMC_FALLBACK]);
  }
  c->stats.pixels += npix;
  if (kernel_ms) cudaEventElapsedTime(kernel_ms, c->k0, c->k1);
  return PM_OK;
}

// A small host-buffer call (npix <= PM_GRAPH_MAX_PIXELS, one-warp grid) as one
// CUDA graph: the caller's arrays are staged through pinned memory, so that
// the graph's copies always use the same addresses and one capture per size
// (and parameter block, tuning and device buffers) serves every later call.
int run_graph_small(pm_ctx* c, int64_t n, const float* spectro, const float* slight, int slight_mode,
                    pm_model* models_out, float* chisq_out, int* iters_out, float* best_fit_out, int* status_out) {
  int rc = stream_resources(c);
  if (rc != PM_OK) return rc;
  if (!c->stage) {
    void* h = nullptr;
    PM_CUDA(cudaHostAlloc(&h, sizeof(SmallStage), cudaHostAllocDefault), "cudaHostAlloc");
    c->stage = static_cast<SmallStage*>(h);
  }
  const size_t kg = PM_GRAPH_MAX_PIXELS;
  for (DevBuf* b : {&c->spectro, &c->slight, &c->spectra})
    if ((rc = b->ensure(kProfMax * kg)) != PM_OK) return rc;
  if ((rc = c->models.ensure(sizeof(pm_model) * kg)) != PM_OK) return rc;
  for (DevBuf* b : {&c->chisq, &c->iters, &c->status})
    if ((rc = b->ensure(sizeof(float) * kg)) != PM_OK) return rc;
  const int nl = c->P.nl;
  const size_t prof = sizeof(float) * 4 * nl;
  SmallStage* st = c->stage;
  HostCtl* hc = c->hc;
  PmStreamQ* q = static_cast<PmStreamQ*>(c->q.p);
  const bool want_spectra = best_fit_out != nullptr, want_status = status_out != nullptr;
  PmJob& job = hc->job;
  std::memset(&job, 0, sizeof job);
  job.npix = n;
  job.spectro = static_cast<const float*>(c->spectro.p);
  job.slight = slight_mode == PM_SLIGHT_PER_PIXEL ? static_cast<const float*>(c->slight.p) : nullptr;
  job.models = static_cast<double*>(c->models.p);
  job.chisq = static_cast<float*>(c->chisq.p);
  job.iters = static_cast<int*>(c->iters.p);
  job.status = want_status ? static_cast<int*>(c->status.p) : nullptr;
  job.spectra = want_spectra ? static_cast<float*>(c->spectra.p) : nullptr;
  job.model_in = nullptr;  // classical estimates in the kernel
  std::memset(&hc->qinit, 0, sizeof hc->qinit);
  hc->qinit.avail = (unsigned long long)n;
  hc->qinit.closed = 1;
  c->gs->ngrids = 1;
  c->gs->g[0] = c->P;
  void* dev[8] = {c->spectro.p, c->slight.p, c->spectra.p, c->models.p, c->chisq.p, c->iters.p, c->status.p, c->q.p};
  const unsigned char* pb = reinterpret_cast<const unsigned char*>(&c->P);

  SmallGraph* G = nullptr;
  for (SmallGraph& g : c->graphs) {
    if (g.exec && g.npix == n && g.slight_mode == slight_mode && g.spectra == want_spectra &&
        g.status == want_status && std::memcmp(&g.tuning, &c->tuning, sizeof g.tuning) == 0 &&
        std::memcmp(g.dev, dev, sizeof dev) == 0 && g.params.size() == sizeof(PmParams) &&
        std::memcmp(g.params.data(), pb, sizeof(PmParams)) == 0) {
      G = &g;
      break;
    }
  }
  if (!G) {
    G = &c->graphs[c->graph_next];
    c->graph_next = (c->graph_next + 1) % kGraphCache;
    if (G->exec) cudaGraphExecDestroy(G->exec);
    G->exec = nullptr;
    cudaStream_t s = c->s_kern;
    PM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed), "graph capture");
    cudaError_t e = cudaMemcpyAsync(c->spectro.p, st->spectro, prof * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && slight_mode == PM_SLIGHT_PER_PIXEL)
      e = cudaMemcpyAsync(c->slight.p, st->slight, prof * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->jobs.p, &hc->job, sizeof(PmJob), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(q, &hc->qinit, sizeof(PmStreamQ), cudaMemcpyHostToDevice, s);
    int krc = PM_OK;
    if (e == cudaSuccess) {
      PmStreamIO sio{};
      sio.q = q;
      sio.jobs = static_cast<const PmJob*>(c->jobs.p);
      sio.jobs_cap = 1;
      sio.wait_limit_ns = 20000000000LL;
      krc = pmk_invert_stream(*c->gs, sio, c->precision, c->tuning.variant, c->tuning.warps_per_block, false, s,
                              c->num_sms, nullptr);
    }
    if (e == cudaSuccess && krc == PM_OK)
      e = cudaMemcpyAsync(st->models, c->models.p, sizeof(pm_model) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && krc == PM_OK)
      e = cudaMemcpyAsync(st->chisq, c->chisq.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && krc == PM_OK)
      e = cudaMemcpyAsync(st->iters, c->iters.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && krc == PM_OK && want_status)
      e = cudaMemcpyAsync(st->status, c->status.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && krc == PM_OK && want_spectra)
      e = cudaMemcpyAsync(st->spectra, c->spectra.p, prof * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && krc == PM_OK)
      e = cudaMemcpyAsync(&hc->qread, q, sizeof(PmStreamQ), cudaMemcpyDeviceToHost, s);
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(s, &graph);
    if (krc != PM_OK) {
      if (graph) cudaGraphDestroy(graph);
      return fail(krc, "%s", pmk_last_cuda_error());
    }
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return cuda_fail(e != cudaSuccess ? e : e2, "graph capture");
    }
    e = cudaGraphInstantiate(&G->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      G->exec = nullptr;
      return cuda_fail(e, "graph instantiate");
    }
    G->npix = n;
    G->slight_mode = slight_mode;
    G->spectra = want_spectra;
    G->status = want_status;
    G->tuning = c->tuning;
    std::memcpy(G->dev, dev, sizeof dev);
    G->params.assign(pb, pb + sizeof(PmParams));
  }
  std::memcpy(st->spectro, spectro, prof * n);
  if (slight_mode == PM_SLIGHT_PER_PIXEL) std::memcpy(st->slight, slight, prof * n);
  PM_CUDA(cudaEventRecord(c->ev_start, c->stream), "event");
  PM_CUDA(cudaStreamWaitEvent(c->s_kern, c->ev_start, 0), "wait");
  PM_CUDA(cudaEventRecord(c->t0, c->s_kern), "event");
  PM_CUDA(cudaGraphLaunch(G->exec, c->s_kern), "graph launch");
  PM_CUDA(cudaEventRecord(c->t1, c->s_kern), "event");
  PM_CUDA(cudaEventRecord(c->ev_done, c->s_kern), "event");
  PM_CUDA(cudaStreamWaitEvent(c->stream, c->ev_done, 0), "wait");
  PM_CUDA(cudaEventSynchronize(c->t1), "graph replay");
  if (hc->qread.err || hc->qread.next < (unsigned long long)n)
    return fail(PM_EIO, "inversion kernel: queue error %llu, %llu of %lld pixels handed out", hc->qread.err,
                hc->qread.next, (long long)n);
  std::memcpy(models_out, st->models, sizeof(pm_model) * n);
  std::memcpy(chisq_out, st->chisq, sizeof(float) * n);
  std::memcpy(iters_out, st->iters, sizeof(int) * n);
  if (want_status) std::memcpy(status_out, st->status, sizeof(int) * n);
  if (want_spectra) std::memcpy(best_fit_out, st->spectra, prof * n);
  float ms = 0;
  cudaEventElapsedTime(&ms, c->t0, c->t1);
  c->stats.kernel_ms = ms;
  c->stats.pixels += n;
  c->stats.iterations += int64_t(hc->qread.ctr[PMC_ITERS]);
  c->stats.accepted += int64_t(hc->qread.ctr[PMC_ACCEPTED]);
  c->stats.eigen_fallbacks += int64_t(hc->qread.ctr[PMC_FALLBACK]);
  c->stats.graph_replays += 1;
  return PM_OK;
}

// One launch over n pixels whose buffers are all device pointers.  One-warp
// grids: the streamed kernel with every pixel published before the launch (the
// same compiled code as the pipelined host-buffer path and the server).
// The classical-estimates-only mode (miter < 0, as NumberOfCycles < 0 in the
// reference, milos.c:399-520): the estimates from the guess with forInitialUse =
// 0 and no NaN fixes, no lm_mils; iterations and chi^2 are 0 (the zero-filled
// vNumIter / vChisqrf that mode writes), status PM_PIX_CLASSICAL, best-fit
// profiles zero.
int run_classical_only(pm_ctx* c, const PmIO& io, float* kernel_ms) {
  TimingEvents ev;
  PM_CUDA(ev.create(), "classical estimates: events");
  cudaEvent_t a = ev.t0, b = ev.t1;
  cudaEventRecord(a, c->stream);
  int rc = c->P.G == 1 ? pmk_classical_prepass(c->P, io.spectro, io.models_out, io.npix, c->stream, c->num_sms,
                                               io.lambda_pix)
                       : pmk_classical_wide(c->P, io, c->stream, c->num_sms);
  cudaEventRecord(b, c->stream);
  if (rc == PM_OK && io.status_out) rc = pmk_fill_int(io.status_out, io.npix, PM_PIX_CLASSICAL, c->stream);
  if (rc != PM_OK) return fail(rc, "%s", pmk_last_cuda_error());
  const size_t n = size_t(io.npix);
  cudaError_t e = cudaMemsetAsync(io.chisq_out, 0, sizeof(float) * n, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(io.iters_out, 0, sizeof(int) * n, c->stream);
  if (e == cudaSuccess && io.spectra_out)
    e = cudaMemsetAsync(io.spectra_out, 0, sizeof(float) * 4 * c->P.nl * n, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess && kernel_ms) e = cudaEventElapsedTime(kernel_ms, a, b);
  if (e != cudaSuccess) return cuda_fail(e, "classical estimates");
  c->stats.pixels += io.npix;
  return PM_OK;
}

int run_invert(pm_ctx* c, PmIO io, float* kernel_ms) {
  if (c->P.miter < 0) return run_classical_only(c, io, kernel_ms);
  if (c->P.G != 1) {
    PM_CUDA(cudaMemsetAsync(io.ctr, 0, sizeof(unsigned long long) * PMC_COUNT, c->stream), "counter reset");
    int rc = pmk_invert(c->P, io, c->precision, c->stream, c->num_sms, kernel_ms);
    if (rc != PM_OK) return fail(rc, "%s", pmk_last_cuda_error());
    unsigned long long h[PMC_COUNT];
    PM_CUDA(cudaMemcpyAsync(h, io.ctr, sizeof h, cudaMemcpyDeviceToHost, c->stream), "counter D2H");
    PM_CUDA(cudaStreamSynchronize(c->stream), "invert kernel");
    c->stats.pixels += io.npix;
    c->stats.iterations += int64_t(h[PMC_ITERS]);
    c->stats.accepted += int64_t(h[PMC_ACCEPTED]);
    c->stats.eigen_fallbacks += int64_t(h[PMC_FALLBACK]);
    return PM_OK;
  }
  int rc = stream_resources(c);
  if (rc != PM_OK) return rc;
  HostCtl* hc = c->hc;
  PmJob& job = hc->job;
  std::memset(&job, 0, sizeof job);
  job.npix = io.npix;
  job.spectro = io.spectro;
  job.slight = io.slight;
  job.models = io.models_out;
  job.chisq = io.chisq_out;
  job.iters = io.iters_out;
  job.status = io.status_out;
  job.spectra = io.spectra_out;
  // every pixel is on the device before the launch: the classical estimates come
  // from a pre-pass launch (the LM kernel reads them through model_in), which
  // keeps their FP64 code out of the LM kernel's instruction stream
  job.model_in = c->P.classical ? io.models_out : nullptr;
  job.lambda = io.lambda_pix;
  std::memset(&hc->qinit, 0, sizeof hc->qinit);
  hc->qinit.avail = (unsigned long long)io.npix;
  hc->qinit.closed = 1;
  PmStreamQ* q = static_cast<PmStreamQ*>(c->q.p);
  PM_CUDA(cudaMemcpyAsync(c->jobs.p, &job, sizeof job, cudaMemcpyHostToDevice, c->stream), "job H2D");
  PM_CUDA(cudaMemcpyAsync(q, &hc->qinit, sizeof hc->qinit, cudaMemcpyHostToDevice, c->stream), "queue H2D");
  c->gs->ngrids = 1;
  c->gs->g[0] = c->P;
  PmStreamIO sio{};
  sio.q = q;
  sio.jobs = static_cast<const PmJob*>(c->jobs.p);
  sio.jobs_cap = 1;
  sio.first_job = 0;
  sio.wait_limit_ns = 20000000000LL;
  PM_CUDA(cudaEventRecord(c->k0, c->stream), "event");
  if (c->P.classical) {
    rc = pmk_classical_prepass(c->P, io.spectro, io.models_out, io.npix, c->stream, c->num_sms, io.lambda_pix);
    if (rc != PM_OK) return fail(rc, "%s", pmk_last_cuda_error());
  }
  rc = pmk_invert_stream(*c->gs, sio, c->precision, c->tuning.variant, c->tuning.warps_per_block, false, c->stream,
                         c->num_sms, nullptr, 0, io.lambda_pix != nullptr);
  if (rc != PM_OK) return fail(rc, "%s", pmk_last_cuda_error());
  PM_CUDA(cudaEventRecord(c->k1, c->stream), "event");
  PM_CUDA(cudaMemcpyAsync(&hc->qread, q, sizeof(PmStreamQ), cudaMemcpyDeviceToHost, c->stream), "queue D2H");
  PM_CUDA(cudaStreamSynchronize(c->stream), "invert kernel");
  if (hc->qread.err || hc->qread.next < (unsigned long long)io.npix)
    return fail(PM_EIO, "inversion kernel: queue error %llu, %llu of %lld pixels handed out", hc->qread.err,
                hc->qread.next, (long long)io.npix);
  if (kernel_ms) cudaEventElapsedTime(kernel_ms, c->k0, c->k1);
  c->stats.pixels += io.npix;
  c->stats.iterations += int64_t(hc->qread.ctr[PMC_ITERS]);
  c->stats.accepted += int64_t(hc->qread.ctr[PMC_ACCEPTED]);
  c->stats.eigen_fallbacks += int64_t(hc->qread.ctr[PMC_FALLBACK]);
  return PM_OK;
}

}  // namespace

namespace {

// pm_invert_batch and pm_invert_batch_grids (lambda: per-pixel wavelengths or
// nullptr).
int invert_impl(pm_ctx* c, int64_t npix, const float* spectro, const double* lambda, const float* slight,
                int slight_mode, const pm_model* guess, pm_model* models_out, float* chisq_out, int* iters_out,
                float* best_fit_out, int* status_out, int mem) {
  if (!c || !spectro || !guess || !models_out || !chisq_out || !iters_out)
    return fail(PM_EINVAL, "pm_invert_batch: NULL argument");
  PmDeviceGuard dg(c->device);
  if (!dg.ok()) return cuda_fail(dg.err, "pm_invert_batch: selecting the context's device", PM_ENODEV);
  if (npix < 0) return fail(PM_EINVAL, "pm_invert_batch: npix < 0");
  if (mem != PM_MEM_HOST && mem != PM_MEM_DEVICE) return fail(PM_EINVAL, "pm_invert_batch: mem=%d", mem);
  if (int rc = check_guess(c->P, guess); rc != PM_OK) return rc;
  const bool ce_only = c->P.miter < 0;  // classical estimates alone: copy, estimate, copy back
  c->stats = pm_stats{};
  if (npix == 0) return PM_OK;
  set_guess(c->P, guess);
  int rc = set_slight(c->P, slight, slight_mode, mem);
  if (rc != PM_OK) return rc;
  const int nl = c->P.nl;
  const size_t prof = sizeof(float) * 4 * nl;
  TimingEvents ev;  // destroyed on every return path
  PM_CUDA(ev.create(), "pm_invert_batch: events");
  cudaEvent_t t0 = ev.t0, t1 = ev.t1;
  cudaEventRecord(t0, c->stream);
  float kms_total = 0;
  if (mem == PM_MEM_DEVICE) {
    PmIO io{};
    io.npix = npix;
    io.spectro = spectro;
    io.slight = slight_mode == PM_SLIGHT_PER_PIXEL ? slight : nullptr;
    io.models_out = reinterpret_cast<double*>(models_out);
    io.chisq_out = chisq_out;
    io.iters_out = iters_out;
    io.spectra_out = best_fit_out;
    io.status_out = status_out;
    io.ctr = static_cast<unsigned long long*>(c->ctr.p);
    io.lambda_pix = lambda;
    rc = run_invert(c, io, &kms_total);
  } else if (!lambda && !ce_only && c->P.G == 1 && c->tuning.graphs && npix <= PM_GRAPH_MAX_PIXELS) {
    rc = run_graph_small(c, npix, spectro, slight, slight_mode, models_out, chisq_out, iters_out, best_fit_out,
                         status_out);
    kms_total = float(c->stats.kernel_ms);
  } else {
    // pixels per resident chunk: the device copies of one chunk's inputs and outputs fit resident_bytes
    const size_t lam_bytes = lambda ? sizeof(double) * nl : 0;  // per pixel
    const size_t per_pixel = prof * (1 + (slight_mode == PM_SLIGHT_PER_PIXEL) + (best_fit_out != nullptr)) +
                             sizeof(pm_model) + sizeof(float) + 2 * sizeof(int) + lam_bytes;
    // wide grids go through two buffer sets (run_wide_pipelined), in at least 8
    // chunks when the cube is large, so that only the first chunk's copy is not
    // hidden behind an inversion; per-pixel grids copy, then launch, chunk by chunk
    const int sets = (c->P.G != 1 && !lambda && !ce_only) ? 2 : 1;
    int64_t chunk = std::min<int64_t>(npix, std::max<int64_t>(32, int64_t(c->resident_bytes / (per_pixel * sets))));
    if (sets == 2 && npix >= 8 * 4096) chunk = std::min<int64_t>(chunk, (npix / 8 + 31) / 32 * 32);
    const int64_t cap = chunk * sets;
    if ((rc = c->spectro.ensure(prof * cap)) != PM_OK) return rc;
    if (slight_mode == PM_SLIGHT_PER_PIXEL && (rc = c->slight.ensure(prof * cap)) != PM_OK) return rc;
    if ((rc = c->models.ensure(sizeof(pm_model) * cap)) != PM_OK) return rc;
    if ((rc = c->chisq.ensure(sizeof(float) * cap)) != PM_OK) return rc;
    if ((rc = c->iters.ensure(sizeof(int) * cap)) != PM_OK) return rc;
    if (best_fit_out && (rc = c->spectra.ensure(prof * cap)) != PM_OK) return rc;
    if (status_out && (rc = c->status.ensure(sizeof(int) * cap)) != PM_OK) return rc;
    if (lambda && (rc = c->lambda.ensure(lam_bytes * chunk)) != PM_OK) return rc;
    if (sets == 2) {
      rc = run_wide_pipelined(c, npix, chunk, spectro, slight, slight_mode, models_out, chisq_out, iters_out,
                              best_fit_out, status_out, &kms_total);
    }
    pm_stats acc{};
    // per-pixel grids take the copy-then-launch path
    const bool streamed = !lambda && !ce_only && c->P.G == 1 && c->tuning.staging_depth > 0;
    for (int64_t p0 = 0; p0 < npix && rc == PM_OK && sets == 1 && streamed; p0 += chunk) {
      const int64_t n = std::min(chunk, npix - p0);
      float kms = 0, tms = 0;
      rc = run_streamed(c, n, spectro + p0 * 4 * nl, slight_mode == PM_SLIGHT_PER_PIXEL ? slight + p0 * 4 * nl : slight,
                        slight_mode, models_out + p0, chisq_out + p0, iters_out + p0,
                        best_fit_out ? best_fit_out + p0 * 4 * nl : nullptr, status_out ? status_out + p0 : nullptr,
                        &kms, &tms);
      kms_total += kms;
    }
    for (int64_t p0 = 0; p0 < npix && rc == PM_OK && sets == 1 && !streamed; p0 += chunk) {
      const int64_t n = std::min(chunk, npix - p0);
      PM_CUDA(cudaMemcpyAsync(c->spectro.p, spectro + p0 * 4 * nl, prof * n, cudaMemcpyHostToDevice, c->stream),
              "spectro H2D");
      if (slight_mode == PM_SLIGHT_PER_PIXEL)
        PM_CUDA(cudaMemcpyAsync(c->slight.p, slight + p0 * 4 * nl, prof * n, cudaMemcpyHostToDevice, c->stream),
                "slight H2D");
      if (lambda)
        PM_CUDA(cudaMemcpyAsync(c->lambda.p, lambda + p0 * nl, lam_bytes * n, cudaMemcpyHostToDevice, c->stream),
                "lambda H2D");
      PmIO io{};
      io.npix = n;
      io.spectro = static_cast<const float*>(c->spectro.p);
      io.slight = slight_mode == PM_SLIGHT_PER_PIXEL ? static_cast<const float*>(c->slight.p) : nullptr;
      io.models_out = static_cast<double*>(c->models.p);
      io.chisq_out = static_cast<float*>(c->chisq.p);
      io.iters_out = static_cast<int*>(c->iters.p);
      io.spectra_out = best_fit_out ? static_cast<float*>(c->spectra.p) : nullptr;
      io.status_out = status_out ? static_cast<int*>(c->status.p) : nullptr;
      io.ctr = static_cast<unsigned long long*>(c->ctr.p);
      io.lambda_pix = lambda ? static_cast<const double*>(c->lambda.p) : nullptr;
      float kms = 0;
      rc = run_invert(c, io, &kms);
      if (rc != PM_OK) break;
      kms_total += kms;
      acc.pixels += c->stats.pixels;
      acc.iterations += c->stats.iterations;
      acc.accepted += c->stats.accepted;
      acc.eigen_fallbacks += c->stats.eigen_fallbacks;
      c->stats = pm_stats{};
      PM_CUDA(cudaMemcpyAsync(models_out + p0, c->models.p, sizeof(pm_model) * n, cudaMemcpyDeviceToHost, c->stream),
              "models D2H");
      PM_CUDA(cudaMemcpyAsync(chisq_out + p0, c->chisq.p, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream),
              "chisq D2H");
      PM_CUDA(cudaMemcpyAsync(iters_out + p0, c->iters.p, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream),
              "iters D2H");
      if (best_fit_out)
        PM_CUDA(cudaMemcpyAsync(best_fit_out + p0 * 4 * nl, c->spectra.p, prof * n, cudaMemcpyDeviceToHost,
                                c->stream),
                "best fit D2H");
      if (status_out)
        PM_CUDA(cudaMemcpyAsync(status_out + p0, c->status.p, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream),
                "status D2H");
    }
    if (!streamed && sets == 1) c->stats = acc;
  }
  cudaEventRecord(t1, c->stream);
  cudaEventSynchronize(t1);
  float tot = 0;
  cudaEventElapsedTime(&tot, t0, t1);
  c->stats.kernel_ms = kms_total;
  c->stats.total_ms = tot;
  if (rc == PM_OK) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pm_invert_batch");
  }
  return rc;
}

}  // namespace

extern "C" int pm_invert_batch(pm_ctx* c, int64_t npix, const float* spectro, const float* slight, int slight_mode,
                               const pm_model* guess, pm_model* models_out, float* chisq_out, int* iters_out,
                               float* best_fit_out, int* status_out, int mem) {
  return invert_impl(c, npix, spectro, nullptr, slight, slight_mode, guess, models_out, chisq_out, iters_out,
                     best_fit_out, status_out, mem);
}

extern "C" int pm_invert_batch_grids(pm_ctx* c, int64_t npix, const float* spectro, const double* lambda,
                                     const float* slight, int slight_mode, const pm_model* guess,
                                     pm_model* models_out, float* chisq_out, int* iters_out, float* best_fit_out,
                                     int* status_out, int mem) {
  if (!lambda) return fail(PM_EINVAL, "pm_invert_batch_grids: lambda is NULL");
  return invert_impl(c, npix, spectro, lambda, slight, slight_mode, guess, models_out, chisq_out, iters_out,
                     best_fit_out, status_out, mem);
}

namespace {

int synth_impl(pm_ctx* c, int64_t npix, const pm_model* models, const double* lambda, const float* slight,
               int slight_mode, float* spectra_out, float* rf_out, int mem) {
  if (!c || !models || !spectra_out) return fail(PM_EINVAL, "pm_synth_batch: NULL argument");
  PmDeviceGuard dg(c->device);
  if (!dg.ok()) return cuda_fail(dg.err, "pm_synth_batch: selecting the context's device", PM_ENODEV);
  if (npix < 0) return fail(PM_EINVAL, "pm_synth_batch: npix < 0");
  if (mem != PM_MEM_HOST && mem != PM_MEM_DEVICE) return fail(PM_EINVAL, "pm_synth_batch: mem=%d", mem);
  if (npix == 0) return PM_OK;
  int rc = set_slight(c->P, slight, slight_mode, mem);
  if (rc != PM_OK) return rc;
  const int nl = c->P.nl, K = c->P.K;
  const size_t prof = sizeof(float) * 4 * nl;
  PmIO io{};
  io.npix = npix;
  if (mem == PM_MEM_DEVICE) {
    io.models_in = reinterpret_cast<const double*>(models);
    io.slight = slight_mode == PM_SLIGHT_PER_PIXEL ? slight : nullptr;
    io.spectra_out = spectra_out;
    io.rf_out = rf_out;
    io.lambda_pix = lambda;
    rc = pmk_synth(c->P, io, c->precision, c->stream);
    if (rc != PM_OK) return fail(rc, "%s", pmk_last_cuda_error());
    PM_CUDA(cudaStreamSynchronize(c->stream), "synth kernel");
    return PM_OK;
  }
  if ((rc = c->models.ensure(sizeof(pm_model) * npix)) != PM_OK) return rc;
  if ((rc = c->spectra.ensure(prof * npix)) != PM_OK) return rc;
  if (rf_out && (rc = c->rf.ensure(prof * K * npix)) != PM_OK) return rc;
  if (slight_mode == PM_SLIGHT_PER_PIXEL && (rc = c->slight.ensure(prof * npix)) != PM_OK) return rc;
  if (lambda && (rc = c->lambda.ensure(sizeof(double) * nl * npix)) != PM_OK) return rc;
  PM_CUDA(cudaMemcpyAsync(c->models.p, models, sizeof(pm_model) * npix, cudaMemcpyHostToDevice, c->stream),
          "models H2D");
  if (lambda)
    PM_CUDA(cudaMemcpyAsync(c->lambda.p, lambda, sizeof(double) * nl * npix, cudaMemcpyHostToDevice, c->stream),
            "lambda H2D");
  io.lambda_pix = lambda ? static_cast<const double*>(c->lambda.p) : nullptr;
  if (slight_mode == PM_SLIGHT_PER_PIXEL)
    PM_CUDA(cudaMemcpyAsync(c->slight.p, slight, prof * npix, cudaMemcpyHostToDevice, c->stream), "slight H2D");
  io.models_in = static_cast<const double*>(c->models.p);
  io.slight = slight_mode == PM_SLIGHT_PER_PIXEL ? static_cast<const float*>(c->slight.p) : nullptr;
  io.spectra_out = static_cast<float*>(c->spectra.p);
  io.rf_out = rf_out ? static_cast<float*>(c->rf.p) : nullptr;
  rc = pmk_synth(c->P, io, c->precision, c->stream);
  if (rc != PM_OK) return fail(rc, "%s", pmk_last_cuda_error());
  PM_CUDA(cudaMemcpyAsync(spectra_out, c->spectra.p, prof * npix, cudaMemcpyDeviceToHost, c->stream), "spectra D2H");
  if (rf_out)
    PM_CUDA(cudaMemcpyAsync(rf_out, c->rf.p, prof * K * npix, cudaMemcpyDeviceToHost, c->stream), "rf D2H");
  PM_CUDA(cudaStreamSynchronize(c->stream), "synth kernel");
  return PM_OK;
}

}  // namespace

extern "C" int pm_synth_batch(pm_ctx* c, int64_t npix, const pm_model* models, const float* slight,
                              int slight_mode, float* spectra_out, float* rf_out, int mem) {
  return synth_impl(c, npix, models, nullptr, slight, slight_mode, spectra_out, rf_out, mem);
}

extern "C" int pm_synth_batch_grids(pm_ctx* c, int64_t npix, const pm_model* models, const double* lambda,
                                    const float* slight, int slight_mode, float* spectra_out, float* rf_out,
                                    int mem) {
  if (!lambda) return fail(PM_EINVAL, "pm_synth_batch_grids: lambda is NULL");
  return synth_impl(c, npix, models, lambda, slight, slight_mode, spectra_out, rf_out, mem);
}

extern "C" int pm_lm_mils(pm_ctx* c, const float* spectro, pm_model* init_model, float* spectra, float* chisqrf,
                          const float* slight, int* iter) {
  if (!c || !spectro || !init_model || !chisqrf || !iter) return fail(PM_EINVAL, "pm_lm_mils: NULL argument");
  pm_model out;
  int it = 0, status = 0;
  float chi = 0;
  const int rc = pm_invert_batch(c, 1, spectro, slight, slight ? PM_SLIGHT_SHARED : PM_SLIGHT_NONE, init_model, &out,
                                 &chi, &it, spectra, &status, PM_MEM_HOST);
  if (rc != PM_OK) return rc;
  *init_model = out;
  *chisqrf = chi;
  *iter = it;
  return status == PM_PIX_NFREE ? -1 : 1;
}

extern "C" int pm_get_tuning(const pm_ctx* c, pm_tuning* out) {
  if (!c || !out) return fail(PM_EINVAL, "pm_get_tuning: NULL argument");
  *out = c->tuning;
  return PM_OK;
}

extern "C" int pm_set_tuning(pm_ctx* c, const pm_tuning* in) {
  if (!c || !in) return fail(PM_EINVAL, "pm_set_tuning: NULL argument");
  if (in->variant < 0 || in->variant > 2) return fail(PM_EINVAL, "pm_set_tuning: variant=%d", in->variant);
  if (in->staging_depth < 0 || in->staging_depth > PM_STAGING_MAX)
    return fail(PM_EINVAL, "pm_set_tuning: staging_depth=%d (0..%d)", in->staging_depth, PM_STAGING_MAX);
  const int w = in->warps_per_block;
  if (in->variant == 2 ? (w != 4 && w != 8 && w != 16) : (w != 1 && w != 2 && w != 4))
    return fail(PM_EINVAL, "pm_set_tuning: warps_per_block=%d (1, 2 or 4; 4, 8 or 16 with variant 2)", w);
  if (in->graphs != 0 && in->graphs != 1) return fail(PM_EINVAL, "pm_set_tuning: graphs=%d (0 or 1)", in->graphs);
  c->tuning = *in;
  return PM_OK;
}

// The autotuner: every candidate inverts the caller's sample through the
// host-buffer entry point (copies + kernel), the fastest median total time wins.
extern "C" int pm_autotune(pm_ctx* c, int64_t npix, const float* spectro, const float* slight, int slight_mode,
                           const pm_model* guess, int reps, pm_tuning* out) {
  if (!c || !spectro || !guess) return fail(PM_EINVAL, "pm_autotune: NULL argument");
  PmDeviceGuard dg(c->device);
  if (!dg.ok()) return cuda_fail(dg.err, "pm_autotune: selecting the context's device", PM_ENODEV);
  if (npix < 1) return fail(PM_EINVAL, "pm_autotune: npix=%lld", (long long)npix);
  reps = std::max(1, std::min(reps, 16));
  // results in pinned host memory, so that the candidates differ only in what they tune
  struct PinnedOut {
    void* p = nullptr;
    ~PinnedOut() {
      if (p) cudaFreeHost(p);
    }
  } out_buf;
  const size_t out_bytes = (sizeof(pm_model) + sizeof(float) + sizeof(int)) * size_t(npix);
  PM_CUDA(cudaHostAlloc(&out_buf.p, out_bytes, cudaHostAllocDefault), "pm_autotune: pinned results");
  pm_model* models = static_cast<pm_model*>(out_buf.p);
  float* chi = reinterpret_cast<float*>(models + npix);
  int* its = reinterpret_cast<int*>(chi + npix);
  std::vector<pm_tuning> cands;
  const bool fp32 = c->precision == PM_PREC_FP32;
  for (int variant : {0, 1, 2}) {
    if (!fp32 && variant != c->tuning.variant) continue;  // the FP64 kernel has one register budget
    for (int wpb : {1, 2, 4, 8, 16}) {
      if ((variant == 2) != (wpb >= 8)) continue;  // lock-step blocks of 8 or 16 warps; 1, 2, 4 otherwise
      for (int depth : {0, 2, 4}) {
        if (c->P.G != 1 && depth != 0) continue;  // multi-warp grids are not streamed
        cands.push_back(pm_tuning{variant, depth, wpb, c->tuning.graphs});
      }
    }
  }
  const pm_tuning saved = c->tuning;
  pm_tuning best = saved;
  double best_ms = 1e300;
  for (const pm_tuning& t : cands) {
    c->tuning = t;
    std::vector<double> ms;
    for (int r = 0; r <= reps; ++r) {
      const int rc = pm_invert_batch(c, npix, spectro, slight, slight_mode, guess, models, chi, its, nullptr,
                                     nullptr, PM_MEM_HOST);
      if (rc != PM_OK) {
        c->tuning = saved;
        return rc;
      }
      if (r > 0) ms.push_back(c->stats.total_ms);  // the first run is a warm-up
    }
    std::sort(ms.begin(), ms.end());
    const double med = ms[ms.size() / 2];
    if (med < best_ms) {
      best_ms = med;
      best = t;
    }
  }
  c->tuning = best;
  c->stats = pm_stats{};
  if (out) *out = best;
  return PM_OK;
}

extern "C" int pm_selftest_stalled_queue(pm_ctx* c, double limit_ms, int* queue_error, double* elapsed_ms) {
  if (!c || !queue_error || !elapsed_ms) return fail(PM_EINVAL, "pm_selftest_stalled_queue: NULL argument");
  PmDeviceGuard dg(c->device);
  if (!dg.ok()) return cuda_fail(dg.err, "pm_selftest_stalled_queue: selecting the context's device", PM_ENODEV);
  if (!(limit_ms > 0 && limit_ms <= 10000)) return fail(PM_EINVAL, "pm_selftest_stalled_queue: limit_ms out of (0, 1e4]");
  if (c->P.G != 1) return fail(PM_ENOTSUP, "pm_selftest_stalled_queue: one-warp grids only");
  int rc = stream_resources(c);
  if (rc != PM_OK) return rc;
  HostCtl* hc = c->hc;
  PmStreamQ* q = static_cast<PmStreamQ*>(c->q.p);
  // an open queue with nothing published and one (never reached) job
  std::memset(&hc->job, 0, sizeof hc->job);
  hc->job.npix = 1;
  std::memset(&hc->qinit, 0, sizeof hc->qinit);
  PM_CUDA(cudaMemcpyAsync(c->jobs.p, &hc->job, sizeof(PmJob), cudaMemcpyHostToDevice, c->s_kern), "job H2D");
  PM_CUDA(cudaMemcpyAsync(q, &hc->qinit, sizeof(PmStreamQ), cudaMemcpyHostToDevice, c->s_kern), "queue H2D");
  c->gs->ngrids = 1;
  c->gs->g[0] = c->P;
  PmStreamIO sio{};
  sio.q = q;
  sio.jobs = static_cast<const PmJob*>(c->jobs.p);
  sio.jobs_cap = 1;
  sio.wait_limit_ns = (long long)(limit_ms * 1e6);
  PM_CUDA(cudaEventRecord(c->k0, c->s_kern), "event");
  rc = pmk_invert_stream(*c->gs, sio, c->precision, c->tuning.variant, c->tuning.warps_per_block, false, c->s_kern,
                         c->num_sms, nullptr);
  if (rc != PM_OK) return fail(rc, "%s", pmk_last_cuda_error());
  PM_CUDA(cudaEventRecord(c->k1, c->s_kern), "event");
  PM_CUDA(cudaMemcpyAsync(&hc->qread, q, sizeof(PmStreamQ), cudaMemcpyDeviceToHost, c->s_kern), "queue D2H");
  PM_CUDA(cudaStreamSynchronize(c->s_kern), "stalled-queue kernel");
  float ms = 0;
  cudaEventElapsedTime(&ms, c->k0, c->k1);
  *queue_error = int(hc->qread.err);
  *elapsed_ms = ms;
  return PM_OK;
}

extern "C" int pm_get_stats(const pm_ctx* c, pm_stats* out) {
  if (!c || !out) return fail(PM_EINVAL, "pm_get_stats: NULL argument");
  *out = c->stats;
  return PM_OK;
}

extern "C" const char* pm_last_error(void) { return g_last_error; }
extern "C" int pm_abi_version(void) { return PMILOS_ABI_VERSION; }
