// pm_stream.cu -- the streamed inversion kernel (a persistent kernel fed while it
// runs: pipelined host-buffer calls and the serving loop) and its launcher.
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
    jp = *reinterpret_cast<const PmJob* const volatile*>(&sm.job);
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
}


// Classical estimates (estimacionesClasicas + the NaN fixes of milos.c:975-983),
// one warp per pixel, written to models as the starting models of the streamed
// kernel when the cube is on the device before the launch.
__global__ void __launch_bounds__(256) classical_prepass_kernel(const __grid_constant__ PmParams P,
                                                                const float* spectro, double* models,
                                                                long long npix, const double* lambda) {
  const int lane = threadIdx.x & 31;
  const bool valid = lane < P.nl;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long pix = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); pix < npix; pix += nwarps) {
    const size_t base = size_t(pix) * 4 * P.nl;
    float O[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) O[s] = valid ? spectro[base + s * P.nl + lane] : 0.0f;
    const double dl = !valid ? 0.0 : (lambda ? lambda[size_t(pix) * P.nl + lane] - P.lambda0 : P.dl[lane]);
    double g[11];
#pragma unroll
    for (int i = 0; i < 11; ++i) g[i] = P.guess[i];
    classical(P, O, lane, valid, dl, g);
    double mine = g[0];
#pragma unroll
    for (int i = 1; i < 11; ++i)
      if (lane == i) mine = g[i];
    if (lane < 11) models[size_t(pix) * 11 + lane] = mine;
  }
}

template <typename R, int KT, int MINB, bool MULTI, bool MAC, bool PIXGRID = false, bool ZM = false>
int launch_invert_stream(const PmGridSet& GS, const PmStreamIO& sio, cudaStream_t st, int num_sms,
                         size_t* smem_out, int wpb, int reserve) {
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

// MAC: the macroturbulence branch compiled in (a grid with a v_mac row).
// pixgrid: per-pixel wavelengths (single-grid launches only).
template <typename R, int KT, bool MAC>
int launch_stream_any(const PmGridSet& GS, const PmStreamIO& sio, cudaStream_t st, int num_sms, int variant,
                      int wpb, bool multi, size_t* smem_out, int reserve, bool pixgrid) {
  if (pixgrid) {
    if (multi) return snprintf(pmk_g_err, sizeof pmk_g_err, "pixel grids: single-grid launches only"), PM_EINVAL;
    if constexpr (sizeof(R) == 4) {
      return variant == 1
                 ? launch_invert_stream<float, KT, 4, false, MAC, true>(GS, sio, st, num_sms, smem_out, wpb, reserve)
                 : launch_invert_stream<float, KT, 3, false, MAC, true>(GS, sio, st, num_sms, smem_out, wpb, reserve);
    } else {
      return launch_invert_stream<double, KT, 1, false, MAC, true>(GS, sio, st, num_sms, smem_out, wpb, reserve);
    }
  }
  if constexpr (sizeof(R) == 4) {
    if (multi) return launch_invert_stream<float, KT, 4, true, MAC>(GS, sio, st, num_sms, smem_out, wpb, reserve);
    return variant == 1 ? launch_invert_stream<float, KT, 4, false, MAC>(GS, sio, st, num_sms, smem_out, wpb, reserve)
                        : launch_invert_stream<float, KT, 3, false, MAC>(GS, sio, st, num_sms, smem_out, wpb, reserve);
  } else {
    return multi ? launch_invert_stream<double, KT, 1, true, MAC>(GS, sio, st, num_sms, smem_out, wpb, reserve)
                 : launch_invert_stream<double, KT, 1, false, MAC>(GS, sio, st, num_sms, smem_out, wpb, reserve);
  }
}

template <typename R>
int launch_stream_k(const PmGridSet& GS, const PmStreamIO& sio, cudaStream_t st, int num_sms, int variant, int wpb,
                    bool multi, size_t* smem_out, int reserve, int K, bool mac, bool pg) {
  // NTERMS 9 never has a v_mac row and 11 always has one (milos.c:152-157)
  if (K == 9) return launch_stream_any<R, 9, false>(GS, sio, st, num_sms, variant, wpb, multi, smem_out, reserve, pg);
  if (K == 10 && mac)
    return launch_stream_any<R, 10, true>(GS, sio, st, num_sms, variant, wpb, multi, smem_out, reserve, pg);
  if (K == 10) return launch_stream_any<R, 10, false>(GS, sio, st, num_sms, variant, wpb, multi, smem_out, reserve, pg);
  if (K == 11) return launch_stream_any<R, 11, true>(GS, sio, st, num_sms, variant, wpb, multi, smem_out, reserve, pg);
  snprintf(pmk_g_err, sizeof pmk_g_err, "nterms=%d has no compiled kernel", K);
  return PM_ENOTSUP;
}


}  // namespace

int pmk_invert_stream(const PmGridSet& GS, const PmStreamIO& sio, int precision, int variant, int warps_per_block,
                      bool multi, void* stream, int num_sms, size_t* smem_out, int reserve_blocks, bool pixgrid) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int wpb = (warps_per_block == 1 || warps_per_block == 2) ? warps_per_block : 4;
  if (GS.ngrids < 1 || GS.ngrids > PMK_MAX_GRIDS || (!multi && GS.ngrids != 1)) {
    snprintf(pmk_g_err, sizeof pmk_g_err, "stream: %d grids", GS.ngrids);
    return PM_EINVAL;
  }
  const int K = GS.g[0].K;
  for (int g = 0; g < GS.ngrids; ++g) {
    if (GS.g[g].G != 1 || GS.g[g].K != K) {
      snprintf(pmk_g_err, sizeof pmk_g_err, "stream: grid %d has nl=%d, nterms=%d (streams take nl <= 32, one nterms)", g,
               GS.g[g].nl, GS.g[g].K);
      return PM_ENOTSUP;
    }
  }
  bool mac = false, zm = false;
  for (int g = 0; g < GS.ngrids; ++g) {
    mac = mac || GS.g[g].mac_row >= 0;
    zm = zm || GS.g[g].n_pi > 1 || GS.g[g].n_sig > 1;
  }
  if (zm) {
    // Zeeman multiplets: one grid, shared wavelengths, no macroturbulence row;
    // the FP32 form with the 128-register budget
    if (multi || pixgrid || mac || K > 10) {
      snprintf(pmk_g_err, sizeof pmk_g_err,
               "Zeeman multiplets: single-grid calls on a shared grid without macroturbulence only");
      return PM_ENOTSUP;
    }
    if (precision == PM_PREC_FP32)
      return K == 9 ? launch_invert_stream<float, 9, 4, false, false, false, true>(GS, sio, st, num_sms, smem_out,
                                                                                    wpb, reserve_blocks)
                    : launch_invert_stream<float, 10, 4, false, false, false, true>(GS, sio, st, num_sms, smem_out,
                                                                                     wpb, reserve_blocks);
    return K == 9 ? launch_invert_stream<double, 9, 1, false, false, false, true>(GS, sio, st, num_sms, smem_out, wpb,
                                                                                   reserve_blocks)
                  : launch_invert_stream<double, 10, 1, false, false, false, true>(GS, sio, st, num_sms, smem_out,
                                                                                    wpb, reserve_blocks);
  }
  if (precision == PM_PREC_FP32)
    return launch_stream_k<float>(GS, sio, st, num_sms, variant, wpb, multi, smem_out, reserve_blocks, K, mac, pixgrid);
  return launch_stream_k<double>(GS, sio, st, num_sms, variant, wpb, multi, smem_out, reserve_blocks, K, mac, pixgrid);
}


int pmk_classical_prepass(const PmParams& P, const float* spectro, double* models, int64_t npix, void* stream,
                          int num_sms, const double* lambda, int threads) {
  if (P.G != 1) {
    snprintf(pmk_g_err, sizeof pmk_g_err, "classical pre-pass: one-warp grids only");
    return PM_EINVAL;
  }
  if (threads < 32 || threads > 256 || threads % 32) {
    snprintf(pmk_g_err, sizeof pmk_g_err, "classical pre-pass: %d threads per block", threads);
    return PM_EINVAL;
  }
  const int warps = threads / 32;
  long long blocks = (npix + warps - 1) / warps;
  if (blocks > (long long)num_sms * 128 / warps) blocks = (long long)num_sms * 128 / warps;
  if (blocks < 1) blocks = 1;
  classical_prepass_kernel<<<unsigned(blocks), threads, 0, static_cast<cudaStream_t>(stream)>>>(P, spectro, models,
                                                                                                 npix, lambda);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "classical launch: %s", cudaGetErrorString(e)), PM_EIO;
  return PM_OK;
}
