// pm_stream.cu -- launches of the streamed inversion kernel (a persistent kernel
// fed while it runs: pipelined host-buffer calls and the serving loop) for
// normal Zeeman triplets, and the classical pre-pass.  Multiplets go to
// pm_stream_zm.cu.
#include "pm_stream_kernel.cuh"

namespace {
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
    // the LM kernels' own instance when they follow (the same code as their
    // in-kernel estimates); the estimates-only branch otherwise
    if (P.miter < 0) classical<true>(P, O, lane, valid, dl, g);
    else classical<false>(P, O, lane, valid, dl, g);
    double mine = g[0];
#pragma unroll
    for (int i = 1; i < 11; ++i)
      if (lane == i) mine = g[i];
    if (lane < 11) models[size_t(pix) * 11 + lane] = mine;
  }
}

// MAC: the macroturbulence branch compiled in (a grid with a v_mac row).
// pixgrid: per-pixel wavelengths (single-grid launches only).
template <typename R, int KT, bool MAC>
int launch_stream_any(const PmGridSet& GS, const PmStreamIO& sio, cudaStream_t st, int num_sms, int variant,
                      int wpb, bool multi, size_t* smem_out, int reserve, bool pixgrid) {
  if (pixgrid) {
    if (multi) return snprintf(pmk_g_err, sizeof pmk_g_err, "pixel grids: single-grid launches only"), PM_EINVAL;
    if constexpr (sizeof(R) == 4) {
      return variant != 0  // 1, or 2 where no lock-step instance exists: the 128-register kernel
                 ? launch_invert_stream<float, KT, 4, false, MAC, true>(GS, sio, st, num_sms, smem_out, wpb, reserve)
                 : launch_invert_stream<float, KT, 3, false, MAC, true>(GS, sio, st, num_sms, smem_out, wpb, reserve);
    } else {
      return launch_invert_stream<double, KT, 1, false, MAC, true>(GS, sio, st, num_sms, smem_out, wpb, reserve);
    }
  }
  if constexpr (sizeof(R) == 4) {
    if constexpr (!MAC && KT <= 10) {
      if (variant == 2) {  // lock-step blocks of wpb warps
        if (multi) {
          if (wpb == 16) return launch_invert_lockstep<float, KT, 16, true, MAC>(GS, sio, st, num_sms, smem_out, reserve);
          if (wpb == 4) return launch_invert_lockstep<float, KT, 4, true, MAC>(GS, sio, st, num_sms, smem_out, reserve);
          return launch_invert_lockstep<float, KT, 8, true, MAC>(GS, sio, st, num_sms, smem_out, reserve);
        }
        if (wpb == 16) return launch_invert_lockstep<float, KT, 16, false, MAC>(GS, sio, st, num_sms, smem_out, reserve);
        if (wpb == 4) return launch_invert_lockstep<float, KT, 4, false, MAC>(GS, sio, st, num_sms, smem_out, reserve);
        return launch_invert_lockstep<float, KT, 8, false, MAC>(GS, sio, st, num_sms, smem_out, reserve);
      }
    }
    if (multi) return launch_invert_stream<float, KT, 4, true, MAC>(GS, sio, st, num_sms, smem_out, wpb, reserve);
    return variant != 0 ? launch_invert_stream<float, KT, 4, false, MAC>(GS, sio, st, num_sms, smem_out, wpb, reserve)
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
  const int wpb = (warps_per_block == 1 || warps_per_block == 2 ||
                   (variant == 2 && (warps_per_block == 8 || warps_per_block == 16)))
                      ? warps_per_block
                      : 4;
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
  if (zm)
    return pmk_invert_stream_zm(GS, sio, precision, wpb, multi, stream, num_sms, smem_out, reserve_blocks, pixgrid,
                                mac);
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
