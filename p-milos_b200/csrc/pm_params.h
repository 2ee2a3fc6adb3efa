// pm_params.h -- launch parameter blocks shared by the host code and the kernels.
//
// Everything that is constant for a run (grid, PSF taps, line data, control
// settings, the initial guess, a shared stray-light profile) travels BY VALUE in
// the kernel parameter block, i.e. in the constant bank: a tap read with a
// compile-time index becomes a constant operand of the FMA that uses it, with no
// load instruction at all.  Per-pixel data travels by pointer in PmIO.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pmilos.h"

// Largest wavelength grid: one thread per wavelength, up to four warps per pixel.
#define PMK_NL 128

struct PmParams {
  int nl;          // wavelengths
  int half;        // nl / 2: PSF centre tap (convolution.c:64)
  int K;           // NTERMS
  int miter;       // < 0: classical estimates alone (NumberOfCycles < 0, milos.c:399-520)
  int nfree_base;  // 4*nl - K (CalculaNfree, lib.c:399-407)
  int logclambda;
  int classical;   // estimacionesClasicas before LM
  int has_psf;
  int solver;      // PM_SOLVE_EIGEN | PM_SOLVE_CHOLESKY
  int slight_mode; // PM_SLIGHT_*
  int want_rf;     // synth kernel: also write response functions
  int n_pi, n_sig;
  int G;           // warps per pixel: 1 (nl <= 32), 2 (nl <= 64) or 4 (nl <= 128)
  int tap_lo, tap_hi;  // PSF support: taps outside [tap_lo, tap_hi] are below 1e-18 of the peak
  int fix[11];
  int zero_row[PM_NTERMS_MAX];  // FijaACeroDerivadasNoNecesarias (milosUtils.c:199-227)
  int ff_row;      // RF row that holds d/d(filling factor), or -1
  int mac_row;     // 9 when RF row 9 is d/d(v_mac) (NTERMS 11, or 10 with alpha fixed), else -1
  double lambda0;
  double dl[PMK_NL];                       // lambda_i - lambda0 [A]
  double nu[3][PM_ZEEMAN_MAX];             // splittings: 0 = pi (NUP), 1 = blue (NUB), 2 = NUB mirrored
  double we[3][PM_ZEEMAN_MAX];             // strengths: WEP, WEB, WER
  double geff, fo;
  double w[4];
  double noise, ilambda, toplim, mu;
  double guess[11];
  double taps_d[PMK_NL];                   // G[j], zero for j >= nl
  float taps_f[PMK_NL];
  double omw_d[PMK_NL];                    // 1 - sum of the taps [tap_lo, tap_hi] that land inside the grid at output k
  float omw_f[PMK_NL];
  float sl_f[4 * PMK_NL];                  // shared stray-light profile [4][nl] (float, as read from the cube)
};

// Work-queue / statistics counters (device memory, zeroed before each launch).
enum { PMC_NEXT = 0, PMC_ITERS = 1, PMC_ACCEPTED = 2, PMC_FALLBACK = 3, PMC_COUNT = 4 };

// ---- streamed inversion (a persistent kernel fed while it runs) ----
// Grids (wavelength grid + line + PSF + settings) one streamed launch serves.
#define PMK_MAX_GRIDS 4
struct PmGridSet {
  int ngrids;
  int pad_;
  PmParams g[PMK_MAX_GRIDS];
};

// Ticket queue in device memory.  next: the next ticket to hand out; avail:
// tickets published (written by the host through the copy engine, after the
// data they cover); closed: nonzero once no more tickets will be published (the
// kernel then ends).  Before a launch on a queue that was closed the host sets
// next = avail (every published ticket has been inverted) and closed = 0.
enum { PMQ_ERR_WAIT = 1, PMQ_ERR_JOB = 2 };
struct PmStreamQ {
  unsigned long long next, avail, closed, err;
  unsigned long long ctr[PMC_COUNT];  // statistics, as PmIO::ctr
};

// One scan (job) of the stream: tickets [t0, t0 + npix) with its own buffers
// (device pointers, layouts as PmIO) and grid.
struct PmJob {
  unsigned long long t0;
  long long npix;
  int grid;
  int pad_;
  const float* spectro;
  const float* slight;      // PM_SLIGHT_PER_PIXEL grids: [npix][4][nl]
  double* models;
  float* chisq;
  int* iters;
  int* status;              // nullable
  float* spectra;           // nullable
  unsigned long long* done; // device counter of finished pixels (zeroed before publication), nullable
  int* host_flag;           // mapped host word set to 1 when the last pixel is done, nullable
  const double* model_in;   // [npix][11] starting models of the classical pre-pass, nullable
  const double* lambda;     // [npix][nl] absolute wavelengths of each pixel (pixel grids), else nullptr
};

static_assert(sizeof(PmGridSet) + 64 <= 32764, "kernel parameter block of the streamed kernel exceeds 32 KB");

struct PmStreamIO {
  PmStreamQ* q;
  const PmJob* jobs;        // ring of jobs_cap descriptors; job k lives in slot k % jobs_cap
  int jobs_cap;
  int pad_;
  long long first_job;      // no ticket left belongs to a job before this one
  long long wait_limit_ns;  // longest wait for a ticket before giving up with PMQ_ERR_WAIT
};

struct PmIO {
  int64_t npix;
  const float* spectro;     // [npix][4][nl]
  const float* slight;      // PM_SLIGHT_PER_PIXEL: [npix][4][nl]
  const double* models_in;  // synth kernel: [npix][11]
  double* models_out;       // [npix][11]
  float* chisq_out;         // [npix]
  int* iters_out;           // [npix]
  float* spectra_out;       // [npix][4][nl] (nullable)
  float* rf_out;            // synth kernel: [npix][4][K][nl] (nullable)
  int* status_out;          // [npix] (nullable)
  unsigned long long* ctr;  // PMC_COUNT counters
  const double* lambda_pix; // [npix][nl] absolute wavelengths of each pixel (nullable: the grid's)
};

// Kernel variants compiled into the library.
enum PmVariant { PMV_FP64 = 0, PMV_FP32 = 1 };

// Host-side launchers (pm_kernels.cu).
int pmk_invert(const PmParams& P, const PmIO& io, int precision, void* stream, int num_sms, float* kernel_ms);
int pmk_synth(const PmParams& P, const PmIO& io, int precision, void* stream);
// Grids of more than 32 wavelengths (pm_wide.cu), called by pmk_invert / pmk_synth.
int pmk_invert_wide(const PmParams& P, const PmIO& io, int precision, void* stream, int num_sms, float* kernel_ms);
int pmk_synth_wide(const PmParams& P, const PmIO& io, int precision, void* stream);
// The classical estimates alone on a wide grid (io.models_out, from the guess).
int pmk_classical_wide(const PmParams& P, const PmIO& io, void* stream, int num_sms);
// n ints of p set to value (stream-ordered).
int pmk_fill_int(int* p, int64_t n, int value, void* stream);
// Their instances for multiplets, macroturbulence and per-pixel grids, by
// precision (pm_wide_x32.cu, pm_wide_x64.cu).
int pmk_invert_wide_x32(const PmParams& P, const PmIO& io, void* stream, int num_sms, float* kernel_ms);
int pmk_invert_wide_x64(const PmParams& P, const PmIO& io, void* stream, int num_sms, float* kernel_ms);
int pmk_synth_wide_x32(const PmParams& P, const PmIO& io, void* stream);
int pmk_synth_wide_x64(const PmParams& P, const PmIO& io, void* stream);
// Classical estimates of npix pixels (one-warp grid) into models [npix][11]:
// the starting models of a launch whose cube is on the device before it starts.
// lambda: [npix][nl] absolute wavelengths of each pixel, or nullptr (the grid's).
// threads: block size (a multiple of 32, at most 256); beside a persistent
// kernel, at most that kernel's block size, so that a block fits in the slot one
// of its blocks leaves free.
int pmk_classical_prepass(const PmParams& P, const float* spectro, double* models, int64_t npix, void* stream,
                          int num_sms, const double* lambda = nullptr, int threads = 256);
// Streamed inversion: every grid of GS has the same nterms and nl <= 32.
// multi: grids differ between jobs (dynamic grid index) rather than one grid.
// reserve_blocks: launch that many fewer blocks than fit, leaving room on the
// SMs for short kernels (the classical pre-pass of newly admitted scans) to run
// beside the persistent kernel.  pixgrid: the jobs carry per-pixel wavelengths
// (PmJob::lambda; one grid, not multi).
int pmk_invert_stream(const PmGridSet& GS, const PmStreamIO& sio, int precision, int variant, int warps_per_block,
                      bool multi, void* stream, int num_sms, size_t* smem_out, int reserve_blocks = 0,
                      bool pixgrid = false);
// The same for a Zeeman multiplet (pm_stream_zm.cu): its own kernel instances, so
// the triplet kernels keep their register budget.  mac: a grid has a v_mac row.
int pmk_invert_stream_zm(const PmGridSet& GS, const PmStreamIO& sio, int precision, int warps_per_block, bool multi,
                         void* stream, int num_sms, size_t* smem_out, int reserve_blocks, bool pixgrid, bool mac);
const char* pmk_last_cuda_error();

// Makes dev the calling thread's current device for the guard's scope and puts
// the caller's back afterwards: every entry point that works on a context or a
// server runs on that object's GPU whatever the caller's thread has selected.
// err is the result of selecting dev; an entry point returns PM_ENODEV when it
// is not cudaSuccess rather than work on whatever device is current.
struct PmDeviceGuard {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit PmDeviceGuard(int dev) {
    err = cudaGetDevice(&prev);
    if (err != cudaSuccess) {
      prev = -1;
      return;
    }
    if (prev == dev) {
      prev = -1;
      return;
    }
    err = cudaSetDevice(dev);
    if (err != cudaSuccess) prev = -1;
  }
  bool ok() const { return err == cudaSuccess; }
  ~PmDeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  PmDeviceGuard(const PmDeviceGuard&) = delete;
  PmDeviceGuard& operator=(const PmDeviceGuard&) = delete;
};

// Host helpers (pm_host.cpp) shared with pm_noalloc.cu.
int pmh_fill_params(const pm_line* L, const pm_config* c, PmParams& P);
void pmh_set_guess(PmParams& P, const pm_model* g);
// The stray-light profile or mode of a grid (host memory), as pm_invert_batch sets it.
int pmh_set_slight(PmParams& P, const float* slight, int mode);
// The NTERMS rule of milos.c:152-157 against the guess's v_mac: PM_OK or PM_EINVAL.
int pmh_check_guess(const PmParams& P, const pm_model* g);
int pmh_fail(int code, const char* msg);
