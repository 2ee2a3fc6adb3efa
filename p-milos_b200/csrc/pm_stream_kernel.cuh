// pm_stream_kernel.cuh -- the streamed inversion kernel template and its
// launcher, shared by the translation units that instantiate it: pm_stream.cu
// (normal Zeeman triplets) and pm_stream_zm.cu (Zeeman multiplets).  Everything
// here has internal linkage; each unit compiles its own instances.
#pragma once
#include "pm_device.cuh"

namespace {
// ---------------------------------------------------------------------------
// Streamed inversion: a persistent kernel fed while it runs.  Pixels are
// tickets; the host publishes tickets in stream order after the data they cover
// has been copied (a copy engine writes PmStreamQ::avail), and appends scans
// ("jobs": a run of tickets with its own buffers and wavelength grid) to a ring
// of descriptors.  A warp takes the next ticket with one atomicAdd and owns it:
// if it is not yet published, the warp waits for its publication, so a ticket
// is never handed out twice nor lost.  The kernel ends when the host closes the
// queue (PmStreamQ::closed, written after the last publication): warps holding
// tickets beyond the final count exit.  Waits are bounded: after wait_limit_ns
// without its ticket a warp sets PMQ_ERR_WAIT and exits.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Next ticket, or -1 when the kernel should exit.
__device__ long long next_ticket(PmStreamQ* q, long long limit_ns) {
  const unsigned long long t = atomicAdd(&q->next, 1ull);
  long long since = -1;
  unsigned sleep = 32;
  while (true) {
    if (t < ld_acquire(&q->avail)) return (long long)t;
    if (ld_acquire(&q->closed)) {
      // closed is written after the last publication: one more look
      return t < ld_acquire(&q->avail) ? (long long)t : -1;
    }
    const long long now = global_ns();
    if (since < 0) since = now;
    if (now - since > limit_ns) {
      atomicExch(&q->err, (unsigned long long)PMQ_ERR_WAIT);
      return -1;
    }
    __nanosleep(sleep);
    sleep = sleep < 2048 ? 2 * sleep : 2048;
  }
}


// The grids a launch serves, by value: all PMK_MAX_GRIDS slots for a server's
// mixed launch, one slot otherwise (a 7 KB rather than 28 KB parameter block).
template <int NG>
struct GridParams {
  int ngrids;
  int pad_;
  PmParams g[NG];
};

// The warp's pixel is finished: count it on its job and, when it was the job's
// last pixel, raise the job's host flag (the server's completion signal).
template <typename R>
__device__ __forceinline__ void job_pixel_done(WarpSmem<R>& sm, int lane) {
  const PmJob* jp = *reinterpret_cast<const PmJob* const volatile*>(&sm.job);
  unsigned long long* done = ld_ptr(&jp->done);
  if (done) {
    __threadfence();  // every lane: its part of this pixel's results before the count
    __syncwarp();
    if (lane == 0) {
      int* flag = ld_ptr(&jp->host_flag);
      const unsigned long long np = __ldcg(reinterpret_cast<const unsigned long long*>(&jp->npix));
      if (atomicAdd(done, 1ull) + 1 == np && flag) {
        __threadfence_system();
        *reinterpret_cast<volatile int*>(flag) = 1;
      }
    }
  }
  __syncwarp();
}

template <typename R, int KT, int MINB, bool MULTI, bool MAC, bool PIXGRID, bool ZM = false>
__global__ void __launch_bounds__(128, MINB) invert_stream_kernel(
    const __grid_constant__ GridParams<MULTI ? PMK_MAX_GRIDS : 1> GS, const PmStreamIO sio) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NG = MULTI ? PMK_MAX_GRIDS : 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  BlockSmem<R>* bs = reinterpret_cast<BlockSmem<R>*>(smem_raw);
  WarpSmem<R>& sm = reinterpret_cast<WarpSmem<R>*>(smem_raw + NG * sizeof(BlockSmem<R>))[warp];
#pragma unroll 1
  for (int g = 0; g < NG && g < GS.ngrids; ++g) load_taps<R>(GS.g[g], bs[g]);
  __syncthreads();
  if (lane == 0) {
    sm.job_k = sio.first_job;
    sm.grid_cur = -1;  // grid of the previous pixel: the padded rows are re-zeroed on a change
  }
  __syncwarp();
  while (true) {
    long long t = 0;
    if (lane == 0) t = next_ticket(sio.q, sio.wait_limit_ns);
    t = __shfl_sync(kFull, t, 0);
    if (t < 0) break;
    // the job of ticket t: jobs are appended in ticket order, so it is at or
    // after this warp's previous one
    const PmJob* jp = nullptr;
    unsigned long long t0 = 0;
    long long k = sm.job_k;
    for (int guard = 0; guard <= sio.jobs_cap; ++guard, ++k) {
      const PmJob* c = sio.jobs + (k % sio.jobs_cap);
      const unsigned long long c0 = __ldcg(&c->t0);
      const unsigned long long cn = __ldcg(reinterpret_cast<const unsigned long long*>(&c->npix));
      if ((unsigned long long)t >= c0 && (unsigned long long)t < c0 + cn) {
        jp = c;
        t0 = c0;
        break;
      }
    }
    if (!jp) {
      if (lane == 0) atomicExch(&sio.q->err, (unsigned long long)PMQ_ERR_JOB);
      break;
    }
    const int gi = MULTI ? __ldcg(&jp->grid) : 0;
    const PmParams& P = GS.g[gi];
    if (gi != sm.grid_cur) {
      for (int e = lane; e < 4 * XSR; e += 32) (&sm.xs[0][0])[e] = R(0);
      __syncwarp();
      if (lane == 0) {
        sm.grid_cur = gi;
        sm.xs_dirty = 0;
      }
    }
    if (lane == 0) {
      sm.job_k = k;
      sm.job = jp;
      sm.pix = (unsigned long long)t - t0;
    }
    __syncwarp();
    invert_pixel<R, KT, MAC, PIXGRID, ZM>(P, bs[gi], sm, lane, sio.q->ctr);
    job_pixel_done(sm, lane);
  }
}


// Lock-step form of the streamed kernel: the W warps of a block advance through
// the LM loop together, one pass at a time, with a block barrier before the
// damped solve (lm_solve; where finished warps take new pixels) and one before
// the synthesis and acceptance test (lm_synth), which the update of an accepted
// step (lm_update) follows directly, so that the block executes one part of the
// loop's code at a time and the warps of an SM sub-partition share its
// instruction cache lines.  A warp draws its next ticket (one atomicAdd) as soon as it
// starts a pixel and starts on that ticket, once it is published, when the pixel
// is finished; it never waits for a publication while other warps of its block
// hold pixels (they would wait for it at the barrier, and in a server the
// publication it waits for may depend on their pixels finishing).  Drawing
// ahead and remembering the last published count and the previous ticket's job
// keep the global-memory round trips of taking a ticket off the block's
// critical path.
// A block none of whose warps holds a pixel sleeps between attempts, up to the
// wait limit (then PMQ_ERR_WAIT), and ends once the queue is closed and
// drained.  MULTI: the launch serves up to PMK_MAX_GRIDS grids (a server's),
// each warp on its pixel's grid.  Per pixel the arithmetic is invert_pixel's.
template <typename R, int KT, int W, bool MULTI, bool MAC, bool PIXGRID, bool ZM = false>
__global__ void __launch_bounds__(32 * W, 16 / W) invert_lockstep_kernel(
    const __grid_constant__ GridParams<MULTI ? PMK_MAX_GRIDS : 1> GS, const PmStreamIO sio) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NG = MULTI ? PMK_MAX_GRIDS : 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  BlockSmem<R>* bs = reinterpret_cast<BlockSmem<R>*>(smem_raw);
  WarpSmem<R>& sm = reinterpret_cast<WarpSmem<R>*>(smem_raw + NG * sizeof(BlockSmem<R>))[warp];
#pragma unroll 1
  for (int g = 0; g < NG && g < GS.ngrids; ++g) load_taps<R>(GS.g[g], bs[g]);
  if (lane == 0) {
    sm.job_k = sio.first_job;
    sm.grid_cur = -1;  // grid of the previous pixel: the padded rows are re-zeroed on a change
  }
  __syncthreads();
  __shared__ int s_stop;
  PixelLM<R> L;
  int gi = 0;
  bool have = false, drained = false;
  long long idle_since = -1;
  unsigned sleep_ns = 32;
  // lane 0's drawn, not yet started ticket (drawn as soon as the previous one is
  // taken, so the atomic's round trip overlaps a pixel's work); the last
  // published count seen and the previous ticket's job live in shared memory
  long long held = -1;
  if (lane == 0) {
    sm.avail_seen = 0;
    sm.job = nullptr;
  }
  __syncwarp();
  while (true) {
    while (!have && !drained) {
      long long t = -1;
      bool dr = false;
      if (lane == 0) {
        if (held < 0) held = (long long)atomicAdd(&sio.q->next, 1ull);
        if ((unsigned long long)held >= sm.avail_seen) sm.avail_seen = ld_acquire(&sio.q->avail);
        if ((unsigned long long)held < sm.avail_seen) {
          t = held;
          held = (long long)atomicAdd(&sio.q->next, 1ull);  // the next one, for the next refill
        } else {
          // closed is written after the last publication: the held ticket is then never published
          dr = ld_acquire(&sio.q->closed) && (unsigned long long)held >= ld_acquire(&sio.q->avail);
        }
      }
      t = __shfl_sync(kFull, t, 0);
      if (t < 0) {
        drained = __shfl_sync(kFull, dr ? 1 : 0, 0) != 0;
        break;
      }
      // the ticket's job: usually the previous ticket's, else walk the ring forward
      int found = 0;
      if (lane == 0) {
        if (sm.job && (unsigned long long)t >= sm.job_t0 && (unsigned long long)t < sm.job_t0 + sm.job_n) {
          found = 1;
        } else {
          long long k = sm.job_k;
          for (int guard = 0; guard <= sio.jobs_cap; ++guard, ++k) {
            const PmJob* c = sio.jobs + (k % sio.jobs_cap);
            const unsigned long long c0 = __ldcg(&c->t0);
            const unsigned long long cn = __ldcg(reinterpret_cast<const unsigned long long*>(&c->npix));
            if ((unsigned long long)t >= c0 && (unsigned long long)t < c0 + cn) {
              sm.job = c;
              sm.job_t0 = c0;
              sm.job_n = cn;
              sm.job_k = k;
              found = 1;
              break;
            }
          }
        }
        if (found) {
          sm.pix = (unsigned long long)t - sm.job_t0;
        } else {
          atomicExch(&sio.q->err, (unsigned long long)PMQ_ERR_JOB);
        }
      }
      if (!__shfl_sync(kFull, found, 0)) {
        drained = true;
        break;
      }
      __syncwarp();
      const PmJob* jp = sm.job;
      gi = MULTI ? __ldcg(&jp->grid) : 0;
      if (gi != sm.grid_cur) {
        for (int e = lane; e < 4 * XSR; e += 32) (&sm.xs[0][0])[e] = R(0);
        __syncwarp();
        if (lane == 0) {
          sm.grid_cur = gi;
          sm.xs_dirty = 0;
        }
      }
      __syncwarp();
      lm_begin<R, PIXGRID>(GS.g[gi], bs[gi], sm, lane, L);
      if (L.finished) {
        lm_end<R>(GS.g[gi], sm, lane, L, sio.q->ctr);
        job_pixel_done(sm, lane);
      } else {
        have = true;
      }
    }
    if (!__syncthreads_or(have)) {
      // no warp of the block holds a pixel: done once every warp has seen the
      // queue closed and drained, else wait for a publication (bounded)
      if (__syncthreads_and(drained)) break;
      if (threadIdx.x == 0) {
        const long long now = global_ns();
        if (idle_since < 0) idle_since = now;
        s_stop = now - idle_since > sio.wait_limit_ns;
        if (s_stop) atomicExch(&sio.q->err, (unsigned long long)PMQ_ERR_WAIT);
      }
      __nanosleep(sleep_ns);
      sleep_ns = sleep_ns < 2048 ? 2 * sleep_ns : 2048;
      __syncthreads();
      if (s_stop) break;
      continue;
    }
    idle_since = -1;
    sleep_ns = 32;
    const PmParams& P = GS.g[gi];
    if (have) lm_solve<R, KT>(P, sm, lane, L);
    __syncthreads();
    // no barrier between the synthesis and the update: a warp whose step was
    // accepted starts its response functions while slower warps finish their
    // synthesis (a barrier here cost 2-5%)
    if (have) lm_synth<R, MAC, PIXGRID, ZM>(P, sm, lane, L);
    if (have) {
      lm_update<R, KT, MAC, PIXGRID, ZM>(P, bs[gi], sm, lane, L);
      if (L.finished) {
        lm_end<R>(P, sm, lane, L, sio.q->ctr);
        job_pixel_done(sm, lane);
        have = false;
      }
    }
  }
}

template <typename R, int KT, int W, bool MULTI, bool MAC, bool PIXGRID = false, bool ZM = false>
int launch_invert_lockstep(const PmGridSet& GS, const PmStreamIO& sio, cudaStream_t st, int num_sms,
                           size_t* smem_out, int reserve) {
  constexpr int threads = 32 * W;
  constexpr int NG = MULTI ? PMK_MAX_GRIDS : 1;
  const size_t smem = NG * sizeof(BlockSmem<R>) + sizeof(WarpSmem<R>) * W;
  if (smem_out) *smem_out = smem;
  auto kern = invert_lockstep_kernel<R, KT, W, MULTI, MAC, PIXGRID, ZM>;
  GridParams<NG> gp;  // copied into the launch
  gp.ngrids = GS.ngrids < NG ? GS.ngrids : NG;
  for (int g = 0; g < gp.ngrids; ++g) gp.g[g] = GS.g[g];
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "%s", cudaGetErrorString(e)), PM_EIO;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (e != cudaSuccess || per_sm < 1) return snprintf(pmk_g_err, sizeof pmk_g_err, "occupancy: %s", cudaGetErrorString(e)), PM_EIO;
  const int blocks = per_sm * num_sms - reserve > 1 ? per_sm * num_sms - reserve : 1;
  kern<<<unsigned(blocks), threads, smem, st>>>(gp, sio);
  e = cudaGetLastError();
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "lock-step launch: %s", cudaGetErrorString(e)), PM_EIO;
  return PM_OK;
}

template <typename R, int KT, int MINB, bool MULTI, bool MAC, bool PIXGRID = false, bool ZM = false>
int launch_invert_stream(const PmGridSet& GS, const PmStreamIO& sio, cudaStream_t st, int num_sms,
                         size_t* smem_out, int wpb, int reserve) {
  if (wpb > 4) wpb = 4;  // the lock-step tunings' block sizes: this kernel takes at most 4 warps per block
  const int threads = 32 * wpb;
  const size_t smem = (MULTI ? PMK_MAX_GRIDS : 1) * sizeof(BlockSmem<R>) + sizeof(WarpSmem<R>) * (threads / 32);
  if (smem_out) *smem_out = smem;
  auto kern = invert_stream_kernel<R, KT, MINB, MULTI, MAC, PIXGRID, ZM>;
  constexpr int NG = MULTI ? PMK_MAX_GRIDS : 1;
  GridParams<NG> gp;  // copied into the launch
  gp.ngrids = GS.ngrids < NG ? GS.ngrids : NG;
  for (int g = 0; g < gp.ngrids; ++g) gp.g[g] = GS.g[g];
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "%s", cudaGetErrorString(e)), PM_EIO;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (e != cudaSuccess || per_sm < 1) return snprintf(pmk_g_err, sizeof pmk_g_err, "occupancy: %s", cudaGetErrorString(e)), PM_EIO;
  const int blocks = per_sm * num_sms - reserve > 1 ? per_sm * num_sms - reserve : 1;
  kern<<<unsigned(blocks), threads, smem, st>>>(gp, sio);
  e = cudaGetLastError();
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "stream launch: %s", cudaGetErrorString(e)), PM_EIO;
  return PM_OK;
}

}  // namespace
