// pm_noalloc.cu -- pm_invert_batch_noalloc: the batched inversion for callers that
// must not allocate GPU memory.
//
// Who needs it.  A host program that keeps its cubes in host memory (like the
// reference's own drivers, which hold every pixel in malloc'd arrays) but runs
// where it may not create device allocations of its own: a process whose device
// memory is reserved up front by another component, a memory-accounted service
// that forbids allocations after start-up, or a real-time acquisition loop that
// cannot afford the latency and possible failure of cudaMalloc/cudaFree on the
// critical path.  pm_invert_batch cannot serve them: its context allocates the
// work-queue counters and, for host buffers, device staging copies.
//
// How.  Everything the call needs on the device beyond the caller's own arrays
// lives in one file-scope static device array, g_noalloc_scratch (about 6.5 MB,
// fixed at build time): the ticket queue with its statistics counters, the job
// descriptor, and staging room for at most PM_NOALLOC_MAX_PIXELS pixels of up to
// 32 wavelengths (observed profiles, a per-pixel stray-light cube, models,
// chi^2, iterations, status, best-fit profiles).  Every GPU that loads the
// library holds this memory until the process exits.  The run constants go in
// the kernel's by-value parameter block, so no context is needed either.  The
// inversion is the streamed kernel of every one-warp call path, with all pixels
// published before the launch.  The call makes no cudaMalloc/cudaFree (nor any
// other allocating call) and creates no CUDA events or streams.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "pm_params.h"

namespace {

constexpr int64_t kMaxPix = PM_NOALLOC_MAX_PIXELS;
constexpr int kMaxNl = PM_NOALLOC_MAX_WAVELENGTHS;
constexpr size_t kProf = sizeof(float) * 4 * kMaxNl;  // one pixel's profiles at the largest grid
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffQueue = 0;
constexpr size_t kOffJob = align256(kOffQueue + sizeof(PmStreamQ));
constexpr size_t kOffSpectro = align256(kOffJob + sizeof(PmJob));
constexpr size_t kOffSlight = align256(kOffSpectro + kMaxPix * kProf);
constexpr size_t kOffModels = align256(kOffSlight + kMaxPix * kProf);
constexpr size_t kOffChisq = align256(kOffModels + kMaxPix * sizeof(pm_model));
constexpr size_t kOffIters = align256(kOffChisq + kMaxPix * sizeof(float));
constexpr size_t kOffStatus = align256(kOffIters + kMaxPix * sizeof(int));
constexpr size_t kOffBest = align256(kOffStatus + kMaxPix * sizeof(int));
constexpr size_t kScratchBytes = align256(kOffBest + kMaxPix * kProf);

}  // namespace

// The scratch.  Host code must not use this name as an address: on the host it
// is a stand-in object, not device memory (a kernel given it would fault, or on
// systems where the GPU can reach host memory, silently use the wrong memory).
// The device address comes from cudaGetSymbolAddress with the device current.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
int g_sms[kMaxDevices] = {};  // set-up done once per device: SM count after the architecture check

// Device address of the scratch on the current device.  The architecture check
// and the SM count are set up on the first call made on a device (with that
// device current); the address itself is looked up on every call
// (cudaGetSymbolAddress allocates nothing), so a context recreated by
// cudaDeviceReset between calls, which reloads the module, gets the new
// address rather than a stale one.
int scratch_for_current_device(unsigned char** out, int* sms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return pmh_fail(PM_ENODEV, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return pmh_fail(PM_ERANGE, "device index beyond 63");
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_sms[dev]) {
      int major = 0, nsm = 0;
      e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return pmh_fail(PM_ENODEV, cudaGetErrorString(e));
      if (major != 10) return pmh_fail(PM_ENODEV, "pm_invert_batch_noalloc: this library is built for sm_100a");
      g_sms[dev] = nsm;
    }
    *sms = g_sms[dev];
  }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) return pmh_fail(PM_EIO, e != cudaSuccess ? cudaGetErrorString(e) : "null symbol");
  *out = static_cast<unsigned char*>(p);
  return PM_OK;
}

int cuda_err(cudaError_t e, const char* what) {
  char msg[256];
  std::snprintf(msg, sizeof msg, "%s: %s", what, cudaGetErrorString(e));
  return pmh_fail(PM_EIO, msg);
}

// An error after work was queued on st: wait for that work (it uses the shared
// scratch) before returning, so that a caller who serialises its calls never
// has two calls' GPU work on the scratch at once.  The first error is kept.
int fail_after_queue(cudaStream_t st, int rc) {
  cudaStreamSynchronize(st);
  return rc;
}

}  // namespace

extern "C" int pm_invert_batch_noalloc(const pm_line* line, const pm_config* cfg, int64_t npix, const float* spectro,
                                       const float* slight, int slight_mode, const pm_model* guess,
                                       pm_model* models_out, float* chisq_out, int* iters_out, float* best_fit_out,
                                       int* status_out, void* stream) {
  if (!line || !cfg || !spectro || !guess || !models_out || !chisq_out || !iters_out)
    return pmh_fail(PM_EINVAL, "pm_invert_batch_noalloc: NULL argument");
  if (npix < 0) return pmh_fail(PM_EINVAL, "pm_invert_batch_noalloc: npix < 0");
  if (npix > kMaxPix) {
    char msg[160];
    std::snprintf(msg, sizeof msg,
                  "pm_invert_batch_noalloc: %lld pixels exceed the static scratch (at most %d pixels per call)",
                  (long long)npix, PM_NOALLOC_MAX_PIXELS);
    return pmh_fail(PM_ERANGE, msg);
  }
  if (cfg->nlambda > kMaxNl) {
    char msg[160];
    std::snprintf(msg, sizeof msg, "pm_invert_batch_noalloc: %d wavelengths exceed the static scratch (at most %d)",
                  cfg->nlambda, kMaxNl);
    return pmh_fail(PM_ERANGE, msg);
  }
  PmParams P;
  int rc = pmh_fill_params(line, cfg, P);
  if (rc != PM_OK) return rc;
  if (P.miter < 0) return pmh_fail(PM_EINVAL, "miter < 0: the LM inversion needs miter >= 0");
  rc = pmh_check_guess(P, guess);
  if (rc != PM_OK) return rc;
  pmh_set_guess(P, guess);
  P.slight_mode = slight_mode;
  if (slight_mode != PM_SLIGHT_NONE) {
    if (!slight) return pmh_fail(PM_EINVAL, "pm_invert_batch_noalloc: slight_mode set but slight is NULL");
    if (P.K < 10) return pmh_fail(PM_EINVAL, "stray light requires nterms >= 10 (filling factor or v_mac inverted)");
    if (slight_mode == PM_SLIGHT_SHARED) {
      for (int i = 0; i < 4 * P.nl; ++i) {
        P.sl_f[i] = slight[i];
      }
    } else if (slight_mode != PM_SLIGHT_PER_PIXEL) {
      return pmh_fail(PM_EINVAL, "pm_invert_batch_noalloc: bad slight_mode");
    }
  }
  if (npix == 0) return PM_OK;
  unsigned char* base = nullptr;
  int sms = 0;
  rc = scratch_for_current_device(&base, &sms);
  if (rc != PM_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t prof = sizeof(float) * 4 * P.nl;
  PmStreamQ* q = reinterpret_cast<PmStreamQ*>(base + kOffQueue);
  PmJob* job_dev = reinterpret_cast<PmJob*>(base + kOffJob);
  cudaError_t e;
  if ((e = cudaMemcpyAsync(base + kOffSpectro, spectro, prof * npix, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail_after_queue(st, cuda_err(e, "spectro H2D"));
  if (slight_mode == PM_SLIGHT_PER_PIXEL &&
      (e = cudaMemcpyAsync(base + kOffSlight, slight, prof * npix, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail_after_queue(st, cuda_err(e, "slight H2D"));
  PmIO io{};
  io.npix = npix;
  io.models_out = reinterpret_cast<double*>(base + kOffModels);
  io.chisq_out = reinterpret_cast<float*>(base + kOffChisq);
  io.iters_out = reinterpret_cast<int*>(base + kOffIters);
  io.status_out = status_out ? reinterpret_cast<int*>(base + kOffStatus) : nullptr;
  io.spectra_out = best_fit_out ? reinterpret_cast<float*>(base + kOffBest) : nullptr;
  // the job and the queue (every ticket published, closed) from this stack
  // frame: a copy from pageable memory has read its source when it returns
  PmJob job{};
  job.npix = npix;
  job.spectro = reinterpret_cast<const float*>(base + kOffSpectro);
  job.slight = slight_mode == PM_SLIGHT_PER_PIXEL ? reinterpret_cast<const float*>(base + kOffSlight) : nullptr;
  job.models = io.models_out;
  job.chisq = io.chisq_out;
  job.iters = io.iters_out;
  job.status = io.status_out;
  job.spectra = io.spectra_out;
  job.model_in = nullptr;  // classical estimates in the kernel, as on every one-warp batch path
  PmStreamQ qinit{};
  qinit.avail = (unsigned long long)npix;
  qinit.closed = 1;
  if ((e = cudaMemcpyAsync(job_dev, &job, sizeof job, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail_after_queue(st, cuda_err(e, "job H2D"));
  if ((e = cudaMemcpyAsync(q, &qinit, sizeof qinit, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail_after_queue(st, cuda_err(e, "queue H2D"));
  PmGridSet gs;
  std::memset(&gs, 0, sizeof gs);
  gs.ngrids = 1;
  gs.g[0] = P;
  PmStreamIO sio{};
  sio.q = q;
  sio.jobs = job_dev;
  sio.jobs_cap = 1;
  sio.first_job = 0;
  sio.wait_limit_ns = 20000000000LL;
  // the launch tuning a context starts with (lock-step blocks of 16 pixels)
  rc = pmk_invert_stream(gs, sio, cfg->precision, 2, 16, false, st, sms, nullptr);
  if (rc != PM_OK) return fail_after_queue(st, pmh_fail(rc, pmk_last_cuda_error()));
  if ((e = cudaMemcpyAsync(models_out, io.models_out, sizeof(pm_model) * npix, cudaMemcpyDeviceToHost, st)) !=
      cudaSuccess)
    return fail_after_queue(st, cuda_err(e, "models D2H"));
  if ((e = cudaMemcpyAsync(chisq_out, io.chisq_out, sizeof(float) * npix, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return fail_after_queue(st, cuda_err(e, "chisq D2H"));
  if ((e = cudaMemcpyAsync(iters_out, io.iters_out, sizeof(int) * npix, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return fail_after_queue(st, cuda_err(e, "iters D2H"));
  if (status_out &&
      (e = cudaMemcpyAsync(status_out, io.status_out, sizeof(int) * npix, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return fail_after_queue(st, cuda_err(e, "status D2H"));
  if (best_fit_out &&
      (e = cudaMemcpyAsync(best_fit_out, io.spectra_out, prof * npix, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return fail_after_queue(st, cuda_err(e, "best fit D2H"));
  PmStreamQ qread{};
  if ((e = cudaMemcpyAsync(&qread, q, sizeof qread, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return fail_after_queue(st, cuda_err(e, "queue D2H"));
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_err(e, "pm_invert_batch_noalloc");
  if (qread.err || qread.next < (unsigned long long)npix)
    return pmh_fail(PM_EIO, "pm_invert_batch_noalloc: the inversion kernel stopped early");
  return PM_OK;
}
