/*
 * pmilos.h -- C ABI of libpmilos_b200.so, the B200 (sm_100a) implementation of
 * P-MILOS's per-pixel Milne-Eddington Stokes inversion.
 *
 * The reference inverts one pixel per call of
 *
 *   int lm_mils(Cuantic *cuantic, PRECISION *wlines, PRECISION *lambda, int nlambda,
 *               float *spectro, int nspectro, Init_Model *initModel, REAL *spectra,
 *               float *chisqrf, REAL *slight, PRECISION toplim, int miter, REAL *weight,
 *               int *fix, REAL *vSigma, REAL sigma, REAL ilambda,
 *               int *INSTRUMENTAL_CONVOLUTION, int *iter, REAL ah, int logclambda);
 *
 * (milosUtils.h:452-455), preceded by estimacionesClasicas (milosUtils.c:287-452) in
 * every per-pixel loop of the drivers (milos.c:958-1009, pmilos.c:1256-1336,
 * :1577-1656, :1851-1930, :2260-2330), with process globals for the line data
 * (create_cuantic), the PSF taps (G) and NTERMS.  This ABI moves those per-run
 * constants into a context and inverts whole slabs of pixels per call.
 *
 * Conventions
 *  - Return codes: 0 on success, negative errno-style values on failure (PM_E*).
 *    Nothing in the library calls exit().
 *  - Buffers are owned by the caller.  Each call says where its buffers live:
 *    PM_MEM_HOST (the library copies through its own device staging buffers;
 *    result arrays in pinned, mapped host memory are written by the kernel
 *    directly where the call streams its cube, see pm_tuning.staging_depth) or
 *    PM_MEM_DEVICE (pointers into this GPU's memory; nothing is copied).
 *  - A context may be used by one host thread at a time; separate contexts are
 *    independent.  All work of a context is ordered on the stream it was created
 *    with (NULL = the legacy default stream).
 *  - Arrays follow the reference's layouts: observed and synthetic profiles are
 *    [pixel][stokes I,Q,U,V][lambda] float32 (utilsFits.c:248, the order lm_mils
 *    consumes); response functions are [pixel][stokes][parameter][lambda]
 *    (me_der.c:243-273); models are pm_model, laid out like Init_Model.
 */
#ifndef PMILOS_H
#define PMILOS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PMILOS_ABI_VERSION 2

/* error codes */
#define PM_OK 0
#define PM_EINVAL (-22)   /* bad argument */
#define PM_ENOMEM (-12)   /* host or device allocation failed */
#define PM_EIO (-5)       /* CUDA runtime error (see pm_last_error) */
#define PM_ENODEV (-19)   /* no usable sm_100 device */
#define PM_ERANGE (-34)   /* size beyond a compiled-in maximum */
#define PM_ENOTSUP (-95)  /* feature outside this implementation's scope */

/* limits */
#define PM_NL_MAX 128      /* wavelengths per profile */
#define PM_NTERMS_MAX 11   /* free parameters */
#define PM_ZEEMAN_MAX 16   /* Zeeman components per group (pi, sigma_b, sigma_r) */

/* buffer residency */
#define PM_MEM_HOST 0
#define PM_MEM_DEVICE 1

/* arithmetic of synthesis, response functions, PSF correlation and normal
 * equations.  The damped solve and the chi^2 acceptance test are FP64 in both. */
#define PM_PREC_FP64 0     /* plain form: the FP64 correctness twin of make use_double=yes */
#define PM_PREC_FP32 1     /* batched form */

/* damped normal-equation solve */
#define PM_SOLVE_DEFAULT 0   /* EIGEN for FP64, CHOLESKY for FP32 */
#define PM_SOLVE_EIGEN 1     /* symmetric eigen-decomposition + pseudo-inverse with the
                                |w| <= 1e-12 cut of mil_svd (milosUtils.c:237-271) */
#define PM_SOLVE_CHOLESKY 2  /* FP64 Cholesky; exactly-zero rows (fixed parameters) give a
                                zero step like the pseudo-inverse; a non-positive pivot
                                falls back to EIGEN for that solve */

/* stray-light modes for pm_invert_batch / pm_synth_batch */
#define PM_SLIGHT_NONE 0     /* no stray light (slight == NULL) */
#define PM_SLIGHT_SHARED 1   /* one [4][nlambda] profile for every pixel */
#define PM_SLIGHT_PER_PIXEL 2/* a [npix][4][nlambda] cube */

/* per-pixel status codes (pm_invert_batch status_out) */
#define PM_PIX_CONVERGED 0   /* relative chi^2 change < toplim or chi^2 < 1e-4 */
#define PM_PIX_LAMBDA 1      /* stopped because the LM damping left [1e-25, 1e7] */
#define PM_PIX_MAXITER 2     /* stopped at miter iterations */
#define PM_PIX_NFREE (-1)    /* no degrees of freedom (lm_mils returns -1) */
#define PM_PIX_NONFINITE (-2)/* a non-finite chi^2 or model was produced */
#define PM_PIX_CLASSICAL 3   /* classical estimates only (pm_config.miter < 0) */

/* Atmosphere model; same field order and types as Init_Model (defines.h:86-98). */
typedef struct pm_model {
  double eta0;  /* line-to-continuum absorption ratio */
  double B;     /* field strength [G] */
  double vlos;  /* line-of-sight velocity [km/s] */
  double dopp;  /* Doppler width [A] */
  double aa;    /* damping */
  double gm;    /* inclination [deg] */
  double az;    /* azimuth [deg] */
  double S0;    /* source function constant */
  double S1;    /* source function gradient */
  double mac;   /* macroturbulence [km/s]; > 1e-4 broadens the profiles */
  double alfa;  /* filling factor */
} pm_model;

/* Spectral line: what create_cuantic (create_cuantic.c:24-294) and wlines[1]
 * provide to the reference.  Strengths and splittings are per Zeeman group
 * (normal triplets and multiplets alike). */
typedef struct pm_line {
  double lambda0;   /* line centre [A] (wlines[1]) */
  int n_pi;         /* components in the pi group (N_PI) */
  int n_sig;        /* components in each sigma group (N_SIG) */
  double nup[PM_ZEEMAN_MAX], nub[PM_ZEEMAN_MAX], nur[PM_ZEEMAN_MAX]; /* splittings (Lande units) */
  double wep[PM_ZEEMAN_MAX], web[PM_ZEEMAN_MAX], wer[PM_ZEEMAN_MAX]; /* strengths */
  double gl, gu, geff; /* Lande factors */
  double fo;        /* relative line strength */
} pm_line;

/* Per-run inversion settings: the control-file fields lm_mils reads
 * (readConfig.c:420-1023) plus this implementation's precision/solver choice. */
typedef struct pm_config {
  int nlambda;            /* 2 .. PM_NL_MAX */
  const double *lambda;   /* [nlambda] absolute wavelengths [A] (vLambda) */
  const double *psf;      /* [nlambda] PSF taps centred at nlambda/2 (G), or NULL */
  double weight[4];       /* Stokes weights (WeightForStokes) */
  double noise;           /* per-point variance (noise = 1/SN^2; lm_mils' sigma) */
  double ilambda;         /* initial LM damping (InitialDiagonalElement) */
  double toplim;          /* relative chi^2 stop (1e-12 in the reference) */
  int miter;              /* max LM iterations (NumberOfCycles > 0); < 0: the classical-estimates-only
                             mode of NumberOfCycles < 0 (milos.c:399-520): estimacionesClasicas from
                             the guess with forInitialUse = 0 (S0 = B_los), no NaN fixes, no LM;
                             iterations and chi^2 0, status PM_PIX_CLASSICAL, best fit zero */
  int fix[11];            /* 1 = parameter is inverted, reference order (defines.h:245) */
  int nterms;             /* NTERMS = 11 - !fix[10] - (guess.mac == 0 && !fix[9]) (milos.c:152-157):
                             9; 10 (filling factor, or v_mac, inverted; or v_mac fixed nonzero); 11.
                             Checked against the guess when one is given (PM_EINVAL) */
  int logclambda;         /* "Diagonal element acceleration" */
  double mu;              /* heliocentric angle cosine (ah) */
  int classical_estimates;/* run estimacionesClasicas + NaN fixes before LM */
  int precision;          /* PM_PREC_FP64 | PM_PREC_FP32 */
  int solver;             /* PM_SOLVE_* */
} pm_config;

/* Run statistics of the last pm_invert_batch on a context. */
typedef struct pm_stats {
  int64_t pixels;
  int64_t iterations;     /* summed over pixels */
  int64_t accepted;       /* LM steps that lowered chi^2 (each re-ran the RFs) */
  int64_t eigen_fallbacks;/* CHOLESKY solves that fell back to EIGEN */
  double kernel_ms;       /* device time of the inversion kernel (CUDA events) */
  double total_ms;        /* device time of the whole call incl. copies */
  int64_t graph_replays;  /* calls served by replaying a captured CUDA graph (pm_tuning.graphs) */
} pm_stats;

typedef struct pm_ctx pm_ctx;

/* Launch choices of a context (what pm_autotune picks; a new context starts with
 * {2, 8, 16, 1}).  No counterpart in the reference, which has no device launches
 * to tune. */
#define PM_STAGING_MAX 64
typedef struct pm_tuning {
  int variant;          /* FP32 kernel of the one-warp grids: 0 = 168 registers per thread (3 blocks of 4
                           warps per SM), 1 = 128 (4 blocks per SM, a few spills), 2 = lock-step blocks
                           (128 registers; the warps of a block run each LM pass together, so they share
                           the instruction-cache lines of its parts; nine or ten free parameters without a
                           v_mac row, one-warp grids; elsewhere 2 runs as 1) */
  int staging_depth;    /* host-buffer calls on grids of <= 32 wavelengths: the cube goes in at most
                           this many pieces, each twice the one before; one persistent launch inverts
                           them as the copy stream publishes each piece (1..PM_STAGING_MAX); 0 = copy
                           everything, then launch.  Output buffers in pinned, mapped host memory
                           (cudaHostAlloc) receive each pixel's results from the kernel directly */
  int warps_per_block;  /* pixels (one warp each) per block of the one-warp kernels: 1, 2 or 4; with
                           variant 2: 4, 8 or 16 */
  int graphs;           /* 1: host-buffer calls of at most PM_GRAPH_MAX_PIXELS pixels on grids of <= 32
                           wavelengths (pm_lm_mils among them) stage through pinned memory and replay a
                           CUDA graph of the whole call, captured once per size; 0: no graphs */
} pm_tuning;
#define PM_GRAPH_MAX_PIXELS 1024

/* ---- host-side precompute (no GPU needed) ---- */

/* Zeeman pattern of one line from its quantum numbers, create_cuantic/Cuanten
 * (create_cuantic.c:60-294); sl, ll, jl / su, lu, ju as readFileCuanticLines
 * (readConfig.c:24-129) decodes them from a LINES entry. */
int pm_line_from_quantum(double lambda0, double sl, double ll, double jl, double su, double lu, double ju,
                         pm_line *out);

/* Gaussian PSF of FWHM [mA] sampled on the grid, fgauss_WL (fgauss.c:79-154). */
int pm_psf_gaussian(double fwhm_ma, int nlambda, const double *lambda, double *taps_out);

/* PSF read from a tabulated profile (offsets [mA], values), linearly
 * interpolated on the grid offsets [mA] and normalised, including the
 * re-centring of milos.c:302-344 / pmilos.c:405-500 and interpolationLinearPSF
 * (milosUtils.c:684-738). */
int pm_psf_interpolate(int nsamples, const double *psf_offsets_ma, const double *psf_values, int nlambda,
                       const double *grid_offsets_ma, double *taps_out);

/* ---- context ---- */

/* Validates cfg, uploads line data, grid and PSF, selects the kernel variant.
 * stream: a cudaStream_t or NULL. */
int pm_ctx_create(const pm_line *line, const pm_config *cfg, void *stream, pm_ctx **out);
int pm_ctx_destroy(pm_ctx *ctx);

/* Invert npix pixels.  Replaces the per-pixel loop of the drivers: for each pixel,
 * start from *guess, apply the classical estimates if cfg->classical_estimates,
 * run the LM loop, and store the model, chi^2 and iteration count like
 * milos.c:998-1006.  best_fit (nullable) receives the profiles of the last
 * synthesis, as lm_mils leaves them in `spectra`.  status (nullable) receives a
 * PM_PIX_* code per pixel.  slight follows slight_mode (PM_SLIGHT_*). */
int pm_invert_batch(pm_ctx *ctx, int64_t npix, const float *spectro, const float *slight, int slight_mode,
                    const pm_model *guess, pm_model *models_out, float *chisq_out, int *iters_out,
                    float *best_fit_out, int *status_out, int mem);

/* Forward synthesis (mil_sinrf) and optionally the response functions (me_der)
 * of npix models, as the reference's synthesis mode (milos.c:601-602) computes
 * them.  rf_out (nullable) is [npix][4][nterms][nlambda].  A model's v_mac broadens
 * its profiles on contexts with nterms >= 10; the v_mac row (row 9 when fix[10] = 0
 * or nterms = 11) is zero for models with v_mac <= 1e-4. */
int pm_synth_batch(pm_ctx *ctx, int64_t npix, const pm_model *models, const float *slight, int slight_mode,
                   float *spectra_out, float *rf_out, int mem);

/* pm_invert_batch / pm_synth_batch with a wavelength grid per pixel: lambda is
 * [npix][nlambda] absolute wavelengths [A] (float64, in the same memory as
 * spectro / models).  The reference documents such grids as a 4-D wavelength
 * FITS file for telecentric and collimated filter set-ups (README "Wavelength
 * grid file (.fits)"); its reader does not load that form
 * (readFitsLambdaToArray, utilsFits.c:749-833), so the definition here is: every
 * pixel is inverted as the reference inverts a cube whose single grid is that
 * pixel's -- synthesis, macroturbulence kernel and classical estimates on the
 * pixel's own wavelengths, the context's PSF taps (sampled at the grid step)
 * for every pixel.  Every grid width (2..PM_NL_MAX); host buffers are copied
 * in, then inverted, chunk by chunk (no pipelining). */
int pm_invert_batch_grids(pm_ctx *ctx, int64_t npix, const float *spectro, const double *lambda,
                          const float *slight, int slight_mode, const pm_model *guess, pm_model *models_out,
                          float *chisq_out, int *iters_out, float *best_fit_out, int *status_out, int mem);
int pm_synth_batch_grids(pm_ctx *ctx, int64_t npix, const pm_model *models, const double *lambda,
                         const float *slight, int slight_mode, float *spectra_out, float *rf_out, int mem);

/* Batch-of-one form of lm_mils for hosts that keep their per-pixel loop: inverts
 * spectro ([4][nlambda], host memory) starting from *init_model (updated in
 * place); spectra (nullable) gets the last synthesis, *chisqrf and *iter the
 * results.  Classical estimates follow cfg->classical_estimates.
 * Returns 1 like lm_mils, -1 when nfree == 0, or a negative PM_E* code. */
int pm_lm_mils(pm_ctx *ctx, const float *spectro, pm_model *init_model, float *spectra, float *chisqrf,
               const float *slight, int *iter);

/* Allocation-free form of pm_invert_batch.  It has no counterpart in the
 * reference.  It is for hosts that keep their cubes in host memory but must not
 * create GPU allocations themselves or through this library (device memory
 * reserved up front by another component, allocation-free real-time loops,
 * memory-accounted services): no context is needed, and the call makes no
 * cudaMalloc/cudaFree or other allocation.  Inputs and outputs are the caller's
 * HOST arrays (same meaning as pm_invert_batch with PM_MEM_HOST); all device-side
 * staging and the work-queue counters live in one static device array built into
 * the library (about 6.5 MB, held on every GPU that loads the library until the
 * process exits), sized for at most PM_NOALLOC_MAX_PIXELS pixels of up to 32
 * wavelengths per call: larger calls fail with PM_ERANGE.  Every call looks up
 * that array's device address on the current device (cudaGetSymbolAddress,
 * which allocates nothing), so a cudaDeviceReset between calls does no harm.
 * The call synchronizes its stream before it returns, on success and on every
 * error after its first copy was queued: do not call it while that stream is
 * being captured into a CUDA graph.  All calls share the one array, and it keeps
 * the last call's contents: calls whose GPU work overlaps (other host threads,
 * other streams) race and must be serialised by the caller.  stream: a
 * cudaStream_t or NULL. */
#define PM_NOALLOC_MAX_PIXELS 4096
#define PM_NOALLOC_MAX_WAVELENGTHS 32
int pm_invert_batch_noalloc(const pm_line *line, const pm_config *cfg, int64_t npix, const float *spectro,
                            const float *slight, int slight_mode, const pm_model *guess, pm_model *models_out,
                            float *chisq_out, int *iters_out, float *best_fit_out, int *status_out, void *stream);

/* ---- cube ingest: FITS spectro cubes into the inversion layout ----
 *
 * The reference reads cubes with CFITSIO and reorders them on the host
 * (readFitsSpectroImage, utilsFits.c:25-368).  Here the host parses the header
 * and the data block goes to the device as stored in the file (big-endian
 * float32); one kernel byte-swaps and permutes it into [pixel][I,Q,U,V][lambda]
 * with pixel = column * rows + row, the reference's generic mapping
 * (utilsFits.c:242-336) for every axis order. */
typedef struct pm_fits_cube {
  int naxis;             /* 4 */
  int64_t naxes[4];      /* NAXIS1..4 */
  int axis_row, axis_col, axis_lambda, axis_stokes;  /* 0-based axis of each role */
  int from_ctype;        /* 1: roles from CTYPE1..4 (HPLN-TAN, HPLT-TAN, WAVE-GRI, STOKES); 0: inferred
                            like the reference (smallest axis Stokes, next smallest wavelength, then
                            rows and columns in axis order) */
  int64_t nrows, ncols, npix;
  int nlambda;
  int64_t data_offset;   /* bytes from the start of the file to the data block */
  int64_t data_bytes;    /* size of the data block */
} pm_fits_cube;

/* Parse the primary header (bytes: the file's first nbytes, at least up to END).
 * PM_ENOTSUP unless BITPIX = -32; PM_EINVAL unless 4 axes with a 4-plane Stokes axis. */
int pm_fits_parse_header(const void *bytes, size_t nbytes, pm_fits_cube *out);
/* Reorder the data block on the device: data_dev holds info->data_bytes bytes as
 * stored in the file, cube_dev receives npix * 4 * nlambda floats.  Device
 * pointers; stream: a cudaStream_t or NULL (asynchronous on it). */
int pm_fits_reorder(const pm_fits_cube *info, const void *data_dev, float *cube_dev, void *stream);

/* ---- serving: continuous batching of spectral scans ----
 *
 * No counterpart in the reference, whose drivers invert one cube per process
 * run.  A server holds up to PM_SERVER_MAX_GRIDS wavelength grids (line, grid,
 * PSF and settings resident on the device; all share nterms and precision) and
 * a device arena of hbm_budget_bytes.  A scheduler thread admits
 * submitted scans in arrival order as arena space and in-flight slots free up:
 * it copies each admitted scan to the device and publishes its pixels to one
 * persistent inversion kernel that is already running, so scans that arrive
 * while others are on the GPU join them; the results of each scan are copied
 * back as soon as its last pixel is done.  Scans on different grids share the
 * launch.  On grids of more than 32 wavelengths each scan is one launch of the
 * wide kernel instead, queued after its copy-in (copies still overlap the
 * inversions of other scans); a server may hold grids of both kinds, and a scan
 * on a wide grid is admitted once the persistent kernel has ended (the scheduler
 * closes it when such a scan is next), then the persistent kernel is launched
 * again for the scans behind it.  Each pixel's arithmetic is the same whatever
 * else is in flight. */
#define PM_SERVER_MAX_GRIDS 4
#define PM_SERVER_MAX_INFLIGHT 256
#define PM_ETIMEDOUT (-110)   /* pm_server_wait: the scan did not finish in time */

typedef struct pm_server pm_server;

typedef struct pm_server_config {
  size_t hbm_budget_bytes;  /* device arena for admitted scans (inputs + results) */
  int max_inflight;         /* scans admitted at once: 1 .. PM_SERVER_MAX_INFLIGHT */
  double linger_ms;         /* an idle persistent kernel exits after this long (relaunched on demand) */
} pm_server_config;

typedef struct pm_scan_info {
  int64_t npix;
  int grid;
  int rc;                   /* PM_OK, or the error that ended the scan */
  double submit_ms, admit_ms, done_ms;  /* host monotonic clock, from server creation */
  int64_t iterations;       /* summed over the scan's pixels */
} pm_scan_info;

typedef struct pm_server_stats {
  int64_t scans_done, pixels_done, kernel_launches;
  double latency_p50_ms, latency_p99_ms, latency_max_ms;  /* submit -> results in host memory */
  double busy_ms;           /* first submit -> last completion */
  size_t arena_peak_bytes;
  int64_t prepass_launches; /* classical-estimate launches apart from the inversion kernel: one per admitted scan
                               on grids wider than 32 wavelengths; 0 on one-warp grids, whose persistent kernel
                               computes the estimates of each pixel it takes */
} pm_server_stats;

/* grids[g], guesses[g]: the settings and initial model of grid g (g < ngrids). */
int pm_server_create(const pm_line *line, const pm_config *const *grids, const pm_model *guesses, int ngrids,
                     const pm_server_config *sc, pm_server **out);
/* Queue a scan of npix pixels on grid `grid`: spectro [npix][4][nl] in host
 * memory (pinned memory lets its copy overlap the kernel); results into the
 * host arrays models_out, chisq_out, iters_out, status_out (nullable).  The
 * arrays must stay valid until the scan is done.  Returns at once with the
 * scan's id; PM_ERANGE if the scan alone exceeds the arena. */
int pm_server_submit(pm_server *srv, int grid, int64_t npix, const float *spectro, pm_model *models_out,
                     float *chisq_out, int *iters_out, int *status_out, uint64_t *id_out);
/* The same for a cube already in this GPU's memory (for instance from
 * pm_fits_reorder): nothing is copied in and the cube takes no arena space; the
 * device array must stay valid until the scan is done. */
int pm_server_submit_device(pm_server *srv, int grid, int64_t npix, const float *spectro_dev, pm_model *models_out,
                            float *chisq_out, int *iters_out, int *status_out, uint64_t *id_out);
/* Block until scan `id` is done (its results are in the host arrays) or
 * timeout_s passes (PM_ETIMEDOUT).  info (nullable) gets its timings. */
int pm_server_wait(pm_server *srv, uint64_t id, double timeout_s, pm_scan_info *info);
/* Stray light of a served grid, as the reference's real-time loop applies its
 * StrayLightFile to every new cube (pmilos.c:2151-2167, :2288-2296):
 * PM_SLIGHT_SHARED, one [4][nlambda] profile for every pixel; PM_SLIGHT_PER_PIXEL,
 * a [npix][4][nlambda] cube in the pixel order of the grid's scans, kept on the
 * device, after which every scan on the grid has exactly npix pixels (else
 * pm_server_submit returns PM_EINVAL); PM_SLIGHT_NONE removes it.  Host memory;
 * the grid's nterms must be >= 10.  Only before the first pm_server_submit
 * (PM_EINVAL afterwards). */
int pm_server_set_slight(pm_server *srv, int grid, const float *slight, int slight_mode, int64_t npix);
int pm_server_get_stats(pm_server *srv, pm_server_stats *out);
/* Finishes every queued scan, then stops the scheduler and frees the device state. */
int pm_server_destroy(pm_server *srv);

int pm_get_tuning(const pm_ctx *ctx, pm_tuning *out);
int pm_set_tuning(pm_ctx *ctx, const pm_tuning *in);

/* Autotuner: inverts npix sample pixels (host buffers, the same call path as
 * pm_invert_batch with PM_MEM_HOST, so copies and kernel are both timed) once per
 * candidate tuning and repetition, and keeps the fastest tuning in the context.
 * Candidates: variants 0 and 1 with warps_per_block {1, 2, 4}, variant 2 with
 * {8, 16}, each with staging_depth {0, 2, 4}.  *out (nullable) receives the
 * choice.  No counterpart in the reference. */
int pm_autotune(pm_ctx *ctx, int64_t npix, const float *spectro, const float *slight, int slight_mode,
                const pm_model *guess, int reps, pm_tuning *out);

/* Self-test of the streamed kernel's bounded wait (no counterpart in the
 * reference): launches it on ctx's grid with a queue that nothing ever
 * publishes to, and a wait limit of limit_ms.  The kernel must give up by itself
 * and report it: *queue_error receives the queue's error word (1 = wait limit
 * reached) and *elapsed_ms the kernel's run time; the context stays usable. */
int pm_selftest_stalled_queue(pm_ctx *ctx, double limit_ms, int *queue_error, double *elapsed_ms);

int pm_get_stats(const pm_ctx *ctx, pm_stats *out);
const char *pm_last_error(void);
int pm_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
