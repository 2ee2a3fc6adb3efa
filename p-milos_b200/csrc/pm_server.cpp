// pm_server.cpp -- the serving loop of include/pmilos.h (pm_server_*): continuous
// batching of spectral scans on one persistent streamed inversion kernel
// (pm_stream.cu), with admission by device-memory budget.
//
// Device state: an arena of hbm_budget_bytes for admitted scans (each scan's
// cube and results), the ticket queue, a ring of job descriptors, per-job done
// counters, and the grids' parameter blocks (kernel parameters).  Host state
// (pinned): the ring's source copies of descriptors and published counts, and
// mapped completion flags the kernel sets when a scan's last pixel is done.
//
// One scheduler thread owns every CUDA call after creation.  Per round it
//  1. admits queued scans in arrival order while a slot and arena space are
//     free: copy the cube (copy stream), write the job descriptor, then
//     publish the scan's tickets (PmStreamQ::avail) -- in that stream order;
//  2. for every scan whose completion flag is set, copies its results back
//     (output stream) and, once that copy is done, frees its arena space and
//     wakes its waiters;
//  3. runs the persistent kernel: launches it when admitted pixels wait and it
//     is stopped, and retires it by closing the queue after linger_ms with
//     nothing in flight (a closed queue ends the kernel once its warps find no
//     published ticket; the next launch reopens the queue at the first
//     unpublished ticket).
// Scans thus join a kernel that is already running, and results leave while
// other scans are still on the GPU.  Grids of more than 32 wavelengths are not
// in the persistent kernel: each admitted scan on one is a launch of the wide
// kernel after its copy-in, and an event on the kernel stream takes the place of
// the completion flag.  A server may hold both kinds of grid; a wide scan is
// admitted only while the persistent kernel is stopped (when one is next in the
// queue the scheduler closes the queue, the kernel ends once its published
// tickets are inverted, and the wide launch follows it on the kernel stream),
// and the persistent kernel is relaunched behind it for the next narrow scans.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "pm_params.h"

namespace {

using Clock = std::chrono::steady_clock;

constexpr int kRing = 4096;  // job descriptor ring: job k lives in slot k % kRing
constexpr size_t kAlign = 256;

size_t round_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

// First-fit allocator over the arena [0, size), 256-byte granules; neighbours
// merge on release.
class Arena {
 public:
  explicit Arena(size_t size) {
    if (size) free_[0] = size;
  }
  bool alloc(size_t bytes, size_t* off) {
    bytes = round_up(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      *off = it->first;
      const size_t rest = it->second - bytes, start = it->first + bytes;
      free_.erase(it);
      if (rest) free_[start] = rest;
      used_ += bytes;
      peak_ = std::max(peak_, used_);
      return true;
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = round_up(bytes);
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t peak() const { return peak_; }

 private:
  std::map<size_t, size_t> free_;
  size_t used_ = 0, peak_ = 0;
};

struct Scan {
  uint64_t id = 0;
  int grid = 0;
  int64_t npix = 0;
  const float* spectro = nullptr;
  bool device_input = false;  // spectro is caller-owned device memory (no copy, no arena space)
  pm_model* models_out = nullptr;
  float* chisq_out = nullptr;
  int* iters_out = nullptr;
  int* status_out = nullptr;
  size_t off = 0, bytes = 0;                       // arena placement
  size_t o_models = 0, o_chisq = 0, o_iters = 0, o_status = 0;
  long long job = -1;
  enum State { QUEUED, ADMITTED, COPYING_OUT, DONE } state = QUEUED;
  cudaEvent_t ev_out = nullptr;
  cudaEvent_t ev_kernel = nullptr;  // grids wider than one warp: the scan's own launch has ended
  pm_scan_info info{};
};

thread_local char g_err[256];

}  // namespace

struct pm_server {
  int device = 0, num_sms = 148, precision = PM_PREC_FP32, variant = 2, ngrids = 0;
  PmGridSet* gs = nullptr;
  pm_server_config sc{};
  size_t prof[PM_SERVER_MAX_GRIDS] = {};
  float* slight_dev[PM_SERVER_MAX_GRIDS] = {};   // PM_SLIGHT_PER_PIXEL grids: the resident cube
  int64_t slight_npix[PM_SERVER_MAX_GRIDS] = {};  // and its pixel count (every scan on the grid has it)
  cudaStream_t s_kern = nullptr, s_copy = nullptr, s_out = nullptr;
  cudaEvent_t ev_kernel = nullptr, ev_reset = nullptr;
  // grids of more than 32 wavelengths: not in the persistent kernel; each
  // admitted scan is one launch of the wide kernel on the kernel stream, after
  // its copy-in (ev_copied), with its pixel and iteration counters in ctr_dev.
  // The persistent kernel serves the other grids (narrow_index: a grid's slot in
  // gs_narrow, the parameter blocks it takes)
  bool wide_grid[PM_SERVER_MAX_GRIDS] = {};
  int narrow_index[PM_SERVER_MAX_GRIDS] = {};
  int nnarrow = 0;
  PmGridSet* gs_narrow = nullptr;
  cudaEvent_t ev_copied = nullptr;
  unsigned long long* ctr_dev = nullptr;
  enum { K_STOPPED, K_RUNNING, K_CLOSING } kstate = K_STOPPED;
  double idle_since = -1;                   // ms; nothing queued or in flight since then
  unsigned long long* reset_host = nullptr; // pinned: [0] first unpublished ticket at a relaunch, [1] zero
  unsigned char* arena_dev = nullptr;
  Arena* arena = nullptr;
  PmStreamQ* q = nullptr;
  PmJob* jobs_dev = nullptr;
  unsigned long long* done_dev = nullptr;
  PmJob* jobs_host = nullptr;               // pinned
  unsigned long long* avail_host = nullptr; // pinned
  unsigned long long* one_host = nullptr;   // pinned word holding 1
  int* flags_host = nullptr;                // mapped pinned
  int* flags_dev = nullptr;
  unsigned long long t_next = 0;      // tickets published
  unsigned long long t_consumed = 0;  // tickets the stopped kernel(s) reached (all inverted)
  long long next_job = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Scan*> queued;
  std::vector<Scan*> active;
  std::map<uint64_t, Scan*> scans;
  uint64_t next_id = 1;
  bool stop = false;
  int error = PM_OK;
  char error_msg[256] = "";
  std::thread worker;
  Clock::time_point t0;
  // statistics
  int64_t launches = 0, prepass_launches = 0, scans_done = 0, pixels_done = 0;
  std::vector<double> latencies;
  double first_submit = -1, last_done = 0;

  double now_ms() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }
  long long oldest_job() const {
    long long k = next_job;
    for (const Scan* s : active) k = std::min(k, s->job);
    return k;
  }
};

namespace {

int sfail(int code, const char* fmt, const char* a = "", const char* b = "") {
  std::snprintf(g_err, sizeof g_err, fmt, a, b);
  return pmh_fail(code, g_err);
}

// An error inside the scheduler: every queued and active scan ends with it.
void fail_all_code(pm_server* s, int code, const char* msg) {
  s->error = code;
  std::snprintf(s->error_msg, sizeof s->error_msg, "%s", msg);
  for (Scan* sc : s->active) {
    sc->info.rc = code;
    sc->state = Scan::DONE;
  }
  for (Scan* sc : s->queued) {
    sc->info.rc = code;
    sc->state = Scan::DONE;
  }
  s->active.clear();
  s->queued.clear();
  s->cv_done.notify_all();
}

void fail_all(pm_server* s, const char* what, cudaError_t e) {
  char msg[256];
  std::snprintf(msg, sizeof msg, "%s: %s", what, cudaGetErrorString(e));
  fail_all_code(s, PM_EIO, msg);
}

// Grids of more than 32 wavelengths: the scan's copy-in on the copy stream, then
// its own launch of the wide kernel (classical estimates included) on the
// kernel stream, then an event the scheduler polls.  Launches run one after
// another on the kernel stream; copies in and out overlap them.
bool admit_wide(pm_server* s, Scan* sc) {
  const size_t prof = s->prof[sc->grid];
  unsigned char* base = s->arena_dev + sc->off;
  const PmParams& P = s->gs->g[sc->grid];
  PmIO io{};
  io.npix = sc->npix;
  io.spectro = sc->device_input ? sc->spectro : reinterpret_cast<const float*>(base);
  io.slight = s->slight_dev[sc->grid];
  io.models_out = reinterpret_cast<double*>(base + sc->o_models);
  io.chisq_out = reinterpret_cast<float*>(base + sc->o_chisq);
  io.iters_out = reinterpret_cast<int*>(base + sc->o_iters);
  io.status_out = reinterpret_cast<int*>(base + sc->o_status);
  io.ctr = s->ctr_dev;
  cudaError_t e = cudaSuccess;
  if (!sc->device_input)
    e = cudaMemcpyAsync(base, sc->spectro, prof * size_t(sc->npix), cudaMemcpyHostToDevice, s->s_copy);
  if (e == cudaSuccess) e = cudaEventRecord(s->ev_copied, s->s_copy);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s->s_kern, s->ev_copied, 0);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->ctr_dev, 0, sizeof(unsigned long long) * PMC_COUNT, s->s_kern);
  if (e == cudaSuccess && !sc->ev_kernel) e = cudaEventCreateWithFlags(&sc->ev_kernel, cudaEventDisableTiming);
  int rc = PM_OK;
  if (e == cudaSuccess) {
    rc = pmk_invert(P, io, s->precision, s->s_kern, s->num_sms, nullptr);
    if (rc == PM_OK) e = cudaEventRecord(sc->ev_kernel, s->s_kern);
  }
  if (e != cudaSuccess || rc != PM_OK) {
    sc->info.rc = rc != PM_OK ? rc : PM_EIO;
    sc->state = Scan::DONE;
    if (rc != PM_OK) fail_all_code(s, rc, pmk_last_cuda_error());
    else fail_all(s, "scan launch", e);
    return false;
  }
  ++s->launches;
  if (P.classical) ++s->prepass_launches;
  sc->job = s->next_job++;  // keeps the in-flight bound of the admission loop
  sc->state = Scan::ADMITTED;
  sc->info.admit_ms = s->now_ms();
  s->active.push_back(sc);
  return true;
}

bool admit(pm_server* s, Scan* sc) {
  if (s->wide_grid[sc->grid]) return admit_wide(s, sc);
  const size_t prof = s->prof[sc->grid];
  const long long k = s->next_job;
  const int slot = int(k % kRing);
  unsigned char* base = s->arena_dev + sc->off;
  PmJob& J = s->jobs_host[slot];
  std::memset(&J, 0, sizeof J);
  J.t0 = s->t_next;
  J.npix = sc->npix;
  J.grid = s->narrow_index[sc->grid];
  J.spectro = sc->device_input ? sc->spectro : reinterpret_cast<const float*>(base);
  J.slight = s->slight_dev[sc->grid];
  J.models = reinterpret_cast<double*>(base + sc->o_models);
  J.chisq = reinterpret_cast<float*>(base + sc->o_chisq);
  J.iters = reinterpret_cast<int*>(base + sc->o_iters);
  J.status = reinterpret_cast<int*>(base + sc->o_status);
  J.done = s->done_dev + slot;
  J.host_flag = s->flags_dev + slot;
  reinterpret_cast<volatile int*>(s->flags_host)[slot] = 0;
  cudaError_t e = cudaMemsetAsync(s->done_dev + slot, 0, sizeof(unsigned long long), s->s_copy);
  if (e == cudaSuccess && !sc->device_input)
    e = cudaMemcpyAsync(base, sc->spectro, prof * size_t(sc->npix), cudaMemcpyHostToDevice, s->s_copy);
  // the classical estimates: computed by the persistent kernel for each pixel
  // it takes (J.model_in stays null), so it fills every block slot and no
  // pre-pass launch has to find room beside it
  if (e == cudaSuccess) e = cudaMemcpyAsync(s->jobs_dev + slot, &J, sizeof J, cudaMemcpyHostToDevice, s->s_copy);
  s->avail_host[slot] = s->t_next + (unsigned long long)sc->npix;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&s->q->avail, &s->avail_host[slot], sizeof(unsigned long long), cudaMemcpyHostToDevice,
                        s->s_copy);
  if (e != cudaSuccess) {
    sc->info.rc = PM_EIO;
    sc->state = Scan::DONE;
    fail_all(s, "scan admission", e);
    return false;
  }
  s->t_next += (unsigned long long)sc->npix;
  s->next_job = k + 1;
  sc->job = k;
  sc->state = Scan::ADMITTED;
  sc->info.admit_ms = s->now_ms();
  s->active.push_back(sc);
  return true;
}

// Launch on a stopped kernel: the queue reopens at the first ticket the
// previous kernel did not reach (it ended only after inverting every published
// ticket), then the kernel starts on the kernel stream after those copies.
bool launch(pm_server* s) {
  s->reset_host[0] = s->t_consumed;
  s->reset_host[1] = 0;
  cudaError_t e = cudaMemcpyAsync(&s->q->next, &s->reset_host[0], sizeof(unsigned long long), cudaMemcpyHostToDevice,
                                  s->s_copy);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&s->q->closed, &s->reset_host[1], sizeof(unsigned long long), cudaMemcpyHostToDevice,
                        s->s_copy);
  if (e == cudaSuccess) e = cudaEventRecord(s->ev_reset, s->s_copy);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s->s_kern, s->ev_reset, 0);
  if (e != cudaSuccess) {
    fail_all(s, "queue reopen", e);
    return false;
  }
  PmStreamIO sio{};
  sio.q = s->q;
  sio.jobs = s->jobs_dev;
  sio.jobs_cap = kRing;
  sio.first_job = s->oldest_job();
  sio.wait_limit_ns = (long long)(std::max(1000.0, 2 * s->sc.linger_ms) * 1e6) + 30000000000LL;
  // the grids of at most 32 wavelengths, as they are now (stray light may have been set)
  s->gs_narrow->ngrids = s->nnarrow;
  for (int g = 0; g < s->ngrids; ++g)
    if (!s->wide_grid[g]) s->gs_narrow->g[s->narrow_index[g]] = s->gs->g[g];
  const int rc = pmk_invert_stream(*s->gs_narrow, sio, s->precision, s->variant, s->variant == 2 ? 16 : 4,
                                   s->nnarrow > 1, s->s_kern, s->num_sms, nullptr, 0);
  if (rc != PM_OK) {
    s->error = rc;
    std::snprintf(s->error_msg, sizeof s->error_msg, "%s", pmk_last_cuda_error());
    for (Scan* sc : s->active) {
      sc->info.rc = rc;
      sc->state = Scan::DONE;
    }
    s->active.clear();
    s->cv_done.notify_all();
    return false;
  }
  cudaEventRecord(s->ev_kernel, s->s_kern);
  s->kstate = pm_server::K_RUNNING;
  s->idle_since = -1;
  ++s->launches;
  return true;
}

// Close the queue: the running kernel ends once its warps find nothing published.
bool close_queue(pm_server* s) {
  const cudaError_t e = cudaMemcpyAsync(&s->q->closed, s->one_host, sizeof(unsigned long long),
                                        cudaMemcpyHostToDevice, s->s_copy);
  if (e != cudaSuccess) {
    fail_all(s, "queue close", e);
    return false;
  }
  s->kstate = pm_server::K_CLOSING;
  return true;
}

void copy_out(pm_server* s, Scan* sc) {
  unsigned char* base = s->arena_dev + sc->off;
  const size_t n = size_t(sc->npix);
  cudaError_t e = cudaMemcpyAsync(sc->models_out, base + sc->o_models, sizeof(pm_model) * n, cudaMemcpyDeviceToHost,
                                  s->s_out);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(sc->chisq_out, base + sc->o_chisq, sizeof(float) * n, cudaMemcpyDeviceToHost, s->s_out);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(sc->iters_out, base + sc->o_iters, sizeof(int) * n, cudaMemcpyDeviceToHost, s->s_out);
  if (e == cudaSuccess && sc->status_out)
    e = cudaMemcpyAsync(sc->status_out, base + sc->o_status, sizeof(int) * n, cudaMemcpyDeviceToHost, s->s_out);
  if (e == cudaSuccess && !sc->ev_out) e = cudaEventCreateWithFlags(&sc->ev_out, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(sc->ev_out, s->s_out);
  if (e != cudaSuccess) return fail_all(s, "scan results", e);
  sc->state = Scan::COPYING_OUT;
}

void finish(pm_server* s, Scan* sc) {
  sc->info.done_ms = s->now_ms();
  sc->info.rc = PM_OK;
  int64_t it = 0;
  for (int64_t i = 0; i < sc->npix; ++i) it += sc->iters_out[i] > 0 ? sc->iters_out[i] : 0;
  sc->info.iterations = it;
  s->arena->release(sc->off, sc->bytes);
  sc->state = Scan::DONE;
  ++s->scans_done;
  s->pixels_done += sc->npix;
  s->latencies.push_back(sc->info.done_ms - sc->info.submit_ms);
  s->last_done = sc->info.done_ms;
}

void serve(pm_server* s) {
  // a new thread starts on device 0: work on the server's GPU, or end every scan
  const cudaError_t dev_err = cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  if (dev_err != cudaSuccess) {
    char msg[200];
    std::snprintf(msg, sizeof msg, "scheduler: selecting the server's device: %s", cudaGetErrorString(dev_err));
    fail_all_code(s, PM_ENODEV, msg);
  }
  while (true) {
    bool progress = false;
    if (s->error == PM_OK) {
      // 1. admission, in arrival order
      while (s->kstate != pm_server::K_CLOSING && !s->queued.empty() &&
             int(s->active.size()) < s->sc.max_inflight && s->next_job - s->oldest_job() < kRing) {
        Scan* sc = s->queued.front();
        // a wide scan's launch follows the persistent kernel on the kernel
        // stream: admitted only while that kernel is stopped (step 3 closes it)
        if (s->wide_grid[sc->grid] && s->kstate != pm_server::K_STOPPED) break;
        size_t off = 0;
        if (!s->arena->alloc(sc->bytes, &off)) break;
        s->queued.pop_front();
        sc->off = off;
        if (!admit(s, sc)) break;
        progress = true;
      }
      // 2. completions
      for (size_t i = 0; i < s->active.size() && s->error == PM_OK;) {
        Scan* sc = s->active[i];
        const int slot = int(sc->job % kRing);
        bool inverted = false;
        if (sc->state == Scan::ADMITTED && s->wide_grid[sc->grid]) {
          const cudaError_t e = cudaEventQuery(sc->ev_kernel);
          if (e == cudaSuccess) inverted = true;
          else if (e != cudaErrorNotReady) fail_all(s, "inversion kernel", e);
        } else if (sc->state == Scan::ADMITTED) {
          inverted = reinterpret_cast<volatile int*>(s->flags_host)[slot] == 1;
        }
        if (s->error != PM_OK) break;
        if (inverted) {
          copy_out(s, sc);
          progress = true;
        }
        if (sc->state == Scan::COPYING_OUT) {
          const cudaError_t e = cudaEventQuery(sc->ev_out);
          if (e == cudaSuccess) {
            finish(s, sc);
            s->active.erase(s->active.begin() + i);
            s->cv_done.notify_all();
            progress = true;
            continue;
          }
          if (e != cudaErrorNotReady) fail_all(s, "scan results", e);
        }
        ++i;
      }
      // 3. the persistent kernel
      if (s->error == PM_OK && s->kstate != pm_server::K_STOPPED) {
        const cudaError_t e = cudaEventQuery(s->ev_kernel);
        if (e == cudaSuccess) {
          // ended: normally after a close; otherwise its wait limit ran out
          PmStreamQ qh{};
          const bool read = cudaMemcpyAsync(&qh, s->q, sizeof qh, cudaMemcpyDeviceToHost, s->s_kern) == cudaSuccess &&
                            cudaStreamSynchronize(s->s_kern) == cudaSuccess;
          if (!read || qh.err || s->kstate != pm_server::K_CLOSING) {
            s->error = PM_EIO;
            std::snprintf(s->error_msg, sizeof s->error_msg, "streamed kernel stopped (queue error %llu)", qh.err);
            for (Scan* sc : s->active) {
              sc->info.rc = PM_EIO;
              sc->state = Scan::DONE;
            }
            s->active.clear();
            s->cv_done.notify_all();
          } else {
            s->kstate = pm_server::K_STOPPED;
            s->t_consumed = s->t_next;
            progress = true;
          }
        } else if (e != cudaErrorNotReady) {
          fail_all(s, "inversion kernel", e);
        }
      }
      bool narrow_pending = false;  // admitted scans of the persistent kernel's grids not yet inverted
      for (const Scan* sc : s->active)
        narrow_pending = narrow_pending || (sc->state == Scan::ADMITTED && !s->wide_grid[sc->grid]);
      if (s->error == PM_OK && s->kstate == pm_server::K_STOPPED) {
        if (narrow_pending && launch(s)) progress = true;
      } else if (s->error == PM_OK && s->kstate == pm_server::K_RUNNING) {
        const bool wide_next = !s->queued.empty() && s->wide_grid[s->queued.front()->grid];
        if (wide_next) {
          // the next scan is on a wide grid: close now, the kernel ends once its
          // published tickets are inverted and the wide launch follows it
          if (close_queue(s)) progress = true;
        } else if (!narrow_pending && s->queued.empty()) {
          const double now = s->now_ms();
          if (s->idle_since < 0) s->idle_since = now;
          else if (now - s->idle_since >= s->sc.linger_ms || s->stop) {
            if (close_queue(s)) progress = true;
          }
        } else {
          s->idle_since = -1;
        }
      }
    }
    if (s->stop && s->queued.empty() && s->active.empty() &&
        (s->kstate == pm_server::K_STOPPED || s->error != PM_OK))
      break;
    if (!progress) {
      if (s->active.empty() && (s->queued.empty() || s->error != PM_OK) &&
          (s->kstate == pm_server::K_STOPPED || s->error != PM_OK)) {
        if (s->stop) break;
        s->cv_work.wait(lk);
      } else {
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(20));
        lk.lock();
      }
    }
  }
}

void release(pm_server* s) {
  PmDeviceGuard dg(s->device);
  if (s->s_copy && s->q && s->one_host && s->kstate != pm_server::K_STOPPED) {
    // a kernel still running (after an error): close the queue so that it ends
    cudaMemcpyAsync(&s->q->closed, s->one_host, sizeof(unsigned long long), cudaMemcpyHostToDevice, s->s_copy);
  }
  for (cudaStream_t st : {s->s_copy, s->s_kern, s->s_out})
    if (st) cudaStreamSynchronize(st);
  for (auto& kv : s->scans) {
    if (kv.second->ev_out) cudaEventDestroy(kv.second->ev_out);
    if (kv.second->ev_kernel) cudaEventDestroy(kv.second->ev_kernel);
    delete kv.second;
  }
  s->scans.clear();
  if (s->ev_kernel) cudaEventDestroy(s->ev_kernel);
  if (s->ev_reset) cudaEventDestroy(s->ev_reset);
  if (s->ev_copied) cudaEventDestroy(s->ev_copied);
  for (cudaStream_t st : {s->s_copy, s->s_kern, s->s_out})
    if (st) cudaStreamDestroy(st);
  for (void* p : {(void*)s->arena_dev, (void*)s->q, (void*)s->jobs_dev, (void*)s->done_dev, (void*)s->ctr_dev})
    if (p) cudaFree(p);
  for (float* p : s->slight_dev)
    if (p) cudaFree(p);
  for (void* p : {(void*)s->jobs_host, (void*)s->avail_host, (void*)s->one_host, (void*)s->flags_host,
                  (void*)s->reset_host})
    if (p) cudaFreeHost(p);
  delete s->arena;
  delete s->gs;
  delete s->gs_narrow;
  delete s;
}

}  // namespace

extern "C" int pm_server_create(const pm_line* line, const pm_config* const* grids, const pm_model* guesses,
                                int ngrids, const pm_server_config* sc, pm_server** out) {
  if (!line || !grids || !guesses || !sc || !out) return sfail(PM_EINVAL, "pm_server_create: NULL argument");
  *out = nullptr;
  if (ngrids < 1 || ngrids > PM_SERVER_MAX_GRIDS) return sfail(PM_EINVAL, "pm_server_create: ngrids out of 1..4");
  if (sc->max_inflight < 1 || sc->max_inflight > PM_SERVER_MAX_INFLIGHT)
    return sfail(PM_EINVAL, "pm_server_create: max_inflight out of 1..256");
  if (sc->hbm_budget_bytes < (size_t(1) << 20)) return sfail(PM_EINVAL, "pm_server_create: budget below 1 MiB");
  if (!(sc->linger_ms >= 0)) return sfail(PM_EINVAL, "pm_server_create: linger_ms < 0");
  pm_server* s = new (std::nothrow) pm_server();
  if (!s) return sfail(PM_ENOMEM, "pm_server_create: out of host memory");
  s->gs = new (std::nothrow) PmGridSet();
  if (!s->gs) {
    delete s;
    return sfail(PM_ENOMEM, "pm_server_create: out of host memory");
  }
  s->sc = *sc;
  s->ngrids = ngrids;
  s->gs->ngrids = ngrids;
  for (int g = 0; g < ngrids; ++g) {
    if (!grids[g]) {
      release(s);
      return sfail(PM_EINVAL, "pm_server_create: grid is NULL");
    }
    int rc = pmh_fill_params(line, grids[g], s->gs->g[g]);
    if (rc != PM_OK) {
      release(s);
      return rc;
    }
    rc = pmh_check_guess(s->gs->g[g], &guesses[g]);
    if (rc != PM_OK) {
      release(s);
      return rc;
    }
    pmh_set_guess(s->gs->g[g], &guesses[g]);
    const PmParams& P = s->gs->g[g];
    if (P.miter < 0) {
      release(s);
      return sfail(PM_EINVAL, "pm_server_create: miter < 0 (classical estimates only) is not served");
    }
    s->wide_grid[g] = P.G != 1;
    if (!s->wide_grid[g]) s->narrow_index[g] = s->nnarrow++;
    if (grids[g]->precision != grids[0]->precision || P.K != s->gs->g[0].K) {
      release(s);
      return sfail(PM_EINVAL, "pm_server_create: grids differ in precision or nterms");
    }
    s->prof[g] = sizeof(float) * 4 * size_t(P.nl);
  }
  s->precision = grids[0]->precision;
  s->gs_narrow = new (std::nothrow) PmGridSet();
  if (!s->gs_narrow) {
    release(s);
    return sfail(PM_ENOMEM, "pm_server_create: out of host memory");
  }
  if (const char* v = std::getenv("PMILOS_VARIANT")) s->variant = std::atoi(v) >= 0 && std::atoi(v) <= 2 ? std::atoi(v) : 2;
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDevice(&s->device);
  if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, s->device);
  if (e != cudaSuccess || prop.major != 10) {
    release(s);
    return sfail(PM_ENODEV, "pm_server_create: no sm_100 device");
  }
  s->num_sms = prop.multiProcessorCount;
  void* p = nullptr;
#define SRV_CUDA(call, what)                                                   \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      release(s);                                                              \
      return sfail(e_ == cudaErrorMemoryAllocation ? PM_ENOMEM : PM_EIO, "%s: %s", what, cudaGetErrorString(e_)); \
    }                                                                          \
  } while (0)
  SRV_CUDA(cudaStreamCreateWithFlags(&s->s_kern, cudaStreamNonBlocking), "stream");
  SRV_CUDA(cudaStreamCreateWithFlags(&s->s_copy, cudaStreamNonBlocking), "stream");
  SRV_CUDA(cudaStreamCreateWithFlags(&s->s_out, cudaStreamNonBlocking), "stream");
  SRV_CUDA(cudaEventCreateWithFlags(&s->ev_kernel, cudaEventDisableTiming), "event");
  SRV_CUDA(cudaEventCreateWithFlags(&s->ev_reset, cudaEventDisableTiming), "event");
  SRV_CUDA(cudaEventCreateWithFlags(&s->ev_copied, cudaEventDisableTiming), "event");
  SRV_CUDA(cudaMalloc(&p, sizeof(unsigned long long) * PMC_COUNT), "counters");
  s->ctr_dev = static_cast<unsigned long long*>(p);
  SRV_CUDA(cudaMalloc(&p, sc->hbm_budget_bytes), "arena (hbm_budget_bytes)");
  s->arena_dev = static_cast<unsigned char*>(p);
  s->arena = new (std::nothrow) Arena(sc->hbm_budget_bytes);
  SRV_CUDA(cudaMalloc(&p, sizeof(PmStreamQ)), "queue");
  s->q = static_cast<PmStreamQ*>(p);
  SRV_CUDA(cudaMemset(s->q, 0, sizeof(PmStreamQ)), "queue");
  SRV_CUDA(cudaMalloc(&p, sizeof(PmJob) * kRing), "job ring");
  s->jobs_dev = static_cast<PmJob*>(p);
  SRV_CUDA(cudaMemset(s->jobs_dev, 0, sizeof(PmJob) * kRing), "job ring");
  SRV_CUDA(cudaMalloc(&p, sizeof(unsigned long long) * kRing), "done counters");
  s->done_dev = static_cast<unsigned long long*>(p);
  SRV_CUDA(cudaHostAlloc(&p, sizeof(PmJob) * kRing, cudaHostAllocDefault), "pinned jobs");
  s->jobs_host = static_cast<PmJob*>(p);
  SRV_CUDA(cudaHostAlloc(&p, sizeof(unsigned long long) * kRing, cudaHostAllocDefault), "pinned counts");
  s->avail_host = static_cast<unsigned long long*>(p);
  SRV_CUDA(cudaHostAlloc(&p, sizeof(unsigned long long), cudaHostAllocDefault), "pinned word");
  s->one_host = static_cast<unsigned long long*>(p);
  *s->one_host = 1;
  SRV_CUDA(cudaHostAlloc(&p, 2 * sizeof(unsigned long long), cudaHostAllocDefault), "pinned words");
  s->reset_host = static_cast<unsigned long long*>(p);
  SRV_CUDA(cudaHostAlloc(&p, sizeof(int) * kRing, cudaHostAllocMapped), "mapped flags");
  s->flags_host = static_cast<int*>(p);
  std::memset(s->flags_host, 0, sizeof(int) * kRing);
  SRV_CUDA(cudaHostGetDevicePointer(&p, s->flags_host, 0), "mapped flags");
  s->flags_dev = static_cast<int*>(p);
#undef SRV_CUDA
  if (!s->arena) {
    release(s);
    return sfail(PM_ENOMEM, "pm_server_create: out of host memory");
  }
  s->t0 = Clock::now();
  s->worker = std::thread(serve, s);
  *out = s;
  return PM_OK;
}

namespace {

int submit(pm_server* s, int grid, int64_t npix, const float* spectro, bool device_input, pm_model* models_out,
           float* chisq_out, int* iters_out, int* status_out, uint64_t* id_out) {
  if (!s || !spectro || !models_out || !chisq_out || !iters_out || !id_out)
    return sfail(PM_EINVAL, "pm_server_submit: NULL argument");
  if (grid < 0 || grid >= s->ngrids) return sfail(PM_EINVAL, "pm_server_submit: no such grid");
  if (npix < 1) return sfail(PM_EINVAL, "pm_server_submit: npix < 1");
  if (s->slight_dev[grid] && npix != s->slight_npix[grid])
    return sfail(PM_EINVAL, "pm_server_submit: the grid's stray-light cube has another pixel count");
  Scan* sc = new (std::nothrow) Scan();
  if (!sc) return sfail(PM_ENOMEM, "pm_server_submit: out of host memory");
  const size_t n = size_t(npix);
  sc->grid = grid;
  sc->npix = npix;
  sc->spectro = spectro;
  sc->device_input = device_input;
  sc->models_out = models_out;
  sc->chisq_out = chisq_out;
  sc->iters_out = iters_out;
  sc->status_out = status_out;
  sc->o_models = device_input ? 0 : round_up(s->prof[grid] * n);
  sc->o_chisq = sc->o_models + round_up(sizeof(pm_model) * n);
  sc->o_iters = sc->o_chisq + round_up(sizeof(float) * n);
  sc->o_status = sc->o_iters + round_up(sizeof(int) * n);
  sc->bytes = sc->o_status + round_up(sizeof(int) * n);
  sc->info.npix = npix;
  sc->info.grid = grid;
  if (sc->bytes > s->sc.hbm_budget_bytes) {
    delete sc;
    return sfail(PM_ERANGE, "pm_server_submit: the scan needs more device memory than the whole budget");
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->error != PM_OK) {
      delete sc;
      return pmh_fail(s->error, s->error_msg);
    }
    sc->id = s->next_id++;
    sc->info.submit_ms = s->now_ms();
    if (s->first_submit < 0) s->first_submit = sc->info.submit_ms;
    s->scans[sc->id] = sc;
    s->queued.push_back(sc);
    *id_out = sc->id;
  }
  s->cv_work.notify_one();
  return PM_OK;
}

}  // namespace

extern "C" int pm_server_submit(pm_server* s, int grid, int64_t npix, const float* spectro, pm_model* models_out,
                                float* chisq_out, int* iters_out, int* status_out, uint64_t* id_out) {
  return submit(s, grid, npix, spectro, false, models_out, chisq_out, iters_out, status_out, id_out);
}

extern "C" int pm_server_submit_device(pm_server* s, int grid, int64_t npix, const float* spectro_dev,
                                       pm_model* models_out, float* chisq_out, int* iters_out, int* status_out,
                                       uint64_t* id_out) {
  return submit(s, grid, npix, spectro_dev, true, models_out, chisq_out, iters_out, status_out, id_out);
}

extern "C" int pm_server_set_slight(pm_server* s, int grid, const float* slight, int slight_mode, int64_t npix) {
  if (!s) return sfail(PM_EINVAL, "pm_server_set_slight: NULL server");
  if (grid < 0 || grid >= s->ngrids) return sfail(PM_EINVAL, "pm_server_set_slight: no such grid");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->next_id != 1) return sfail(PM_EINVAL, "pm_server_set_slight: scans were submitted already");
  PmDeviceGuard dg(s->device);
  if (!dg.ok()) return sfail(PM_ENODEV, "pm_server_set_slight: selecting the server's device: %s", cudaGetErrorString(dg.err));
  PmParams& P = s->gs->g[grid];
  if (slight_mode == PM_SLIGHT_PER_PIXEL && (!slight || npix < 1))
    return sfail(PM_EINVAL, "pm_server_set_slight: a per-pixel cube needs slight and npix >= 1");
  const int rc = pmh_set_slight(P, slight, slight_mode);
  if (rc != PM_OK) return rc;
  if (s->slight_dev[grid]) {
    cudaFree(s->slight_dev[grid]);
    s->slight_dev[grid] = nullptr;
    s->slight_npix[grid] = 0;
  }
  if (slight_mode == PM_SLIGHT_PER_PIXEL) {
    const size_t bytes = s->prof[grid] * size_t(npix);
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(p, slight, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      if (p) cudaFree(p);
      P.slight_mode = PM_SLIGHT_NONE;
      return sfail(e == cudaErrorMemoryAllocation ? PM_ENOMEM : PM_EIO, "pm_server_set_slight: %s",
                   cudaGetErrorString(e));
    }
    s->slight_dev[grid] = static_cast<float*>(p);
    s->slight_npix[grid] = npix;
  }
  return PM_OK;
}

extern "C" int pm_server_wait(pm_server* s, uint64_t id, double timeout_s, pm_scan_info* info) {
  if (!s) return sfail(PM_EINVAL, "pm_server_wait: NULL server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->scans.find(id);
  if (it == s->scans.end()) return sfail(PM_EINVAL, "pm_server_wait: unknown scan id (already waited for?)");
  Scan* sc = it->second;
  const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                           std::chrono::duration<double>(std::max(0.0, timeout_s)));
  if (!s->cv_done.wait_until(lk, deadline, [&] { return sc->state == Scan::DONE; }))
    return sfail(PM_ETIMEDOUT, "pm_server_wait: scan not done in time");
  if (info) *info = sc->info;
  const int rc = sc->info.rc;
  s->scans.erase(it);
  if (sc->ev_out) cudaEventDestroy(sc->ev_out);
  if (sc->ev_kernel) cudaEventDestroy(sc->ev_kernel);
  delete sc;
  if (rc != PM_OK) return pmh_fail(rc, s->error_msg);
  return PM_OK;
}

extern "C" int pm_server_get_stats(pm_server* s, pm_server_stats* out) {
  if (!s || !out) return sfail(PM_EINVAL, "pm_server_get_stats: NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof *out);
  out->scans_done = s->scans_done;
  out->pixels_done = s->pixels_done;
  out->kernel_launches = s->launches;
  out->prepass_launches = s->prepass_launches;
  out->arena_peak_bytes = s->arena->peak();
  if (!s->latencies.empty()) {
    std::vector<double> v = s->latencies;
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) {
      const double r = p * double(v.size() - 1);
      const size_t lo = size_t(r), hi = std::min(v.size() - 1, lo + 1);
      return v[lo] + (r - double(lo)) * (v[hi] - v[lo]);
    };
    out->latency_p50_ms = pct(0.50);
    out->latency_p99_ms = pct(0.99);
    out->latency_max_ms = v.back();
  }
  out->busy_ms = s->first_submit >= 0 ? s->last_done - s->first_submit : 0;
  return PM_OK;
}

extern "C" int pm_server_destroy(pm_server* s) {
  if (!s) return PM_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  release(s);
  return PM_OK;
}
