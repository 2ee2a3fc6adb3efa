// pm_kernels.cu -- the one-warp-per-pixel synthesis kernel (grids of up to 32
// wavelengths) and the dispatch of the batch launches: synthesis of any grid,
// inversion of grids wider than one warp (pm_wide.cu).  One-warp inversions run
// the streamed kernel of pm_stream.cu.
#include "pm_device.cuh"

char pmk_g_err[256];

namespace {
template <typename R, int KT, bool ZM>
__global__ void __launch_bounds__(128) synth_kernel(const __grid_constant__ PmParams P, const PmIO io) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  BlockSmem<R>& bs = *reinterpret_cast<BlockSmem<R>*>(smem_raw);
  WarpSmem<R>& sm = warp_smem<R>(smem_raw, warp);
  load_taps<R>(P, bs);
  for (int e = lane; e < 4 * XSR; e += 32) (&sm.xs[0][0])[e] = R(0);
  if (lane == 0) sm.xs_dirty = 0;
  __syncthreads();
  const bool valid = lane < P.nl;
  const int64_t nwarps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t pix = int64_t(blockIdx.x) * (blockDim.x >> 5) + warp; pix < io.npix; pix += nwarps) {
    const size_t base = size_t(pix) * 4 * P.nl;
    const float* sl_pix = slight_of<R>(P, bs, io.slight, base);
    if (lane < 11) sm.model[lane] = io.models_in[size_t(pix) * 11 + lane];
    __syncwarp();
    const double dl = !valid ? 0.0 : (io.lambda_pix ? io.lambda_pix[size_t(pix) * P.nl + lane] - P.lambda0 : P.dl[lane]);
    R S[4], Su[4];
    synthesize<R, (KT >= 10), ZM>(P, sm, sm.model, sl_pix, lane, valid, dl, S, Su);
    if (valid) {
#pragma unroll
      for (int s = 0; s < 4; ++s) io.spectra_out[base + s * P.nl + lane] = float(S[s]);
    }
    if (io.rf_out) {
      R d[KT][4];
      response_rows<R, KT, (KT >= 10), ZM>(P, bs, sm, lane, valid, sm.model, dl, Su, sl_pix, d);
      __syncwarp();
      if (valid) {
        const size_t rb = size_t(pix) * 4 * KT * P.nl;
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
          for (int r = 0; r < KT; ++r) io.rf_out[rb + (size_t(s) * KT + r) * P.nl + lane] = float(d[r][s]);
      }
    }
    __syncwarp();
  }
}


template <typename R, int KT, bool ZM>
int launch_synth(const PmParams& P, const PmIO& io, cudaStream_t st) {
  const int threads = 128;
  const size_t smem = sizeof(BlockSmem<R>) + sizeof(WarpSmem<R>) * (threads / 32);
  auto kern = synth_kernel<R, KT, ZM>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "%s", cudaGetErrorString(e)), PM_EIO;
  int64_t blocks = (io.npix + 3) / 4;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  kern<<<unsigned(blocks), threads, smem, st>>>(P, io);
  e = cudaGetLastError();
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "synth launch: %s", cudaGetErrorString(e)), PM_EIO;
  return PM_OK;
}


template <typename R, int KT>
int launch_synth_any(const PmParams& P, const PmIO& io, cudaStream_t st) {
  if (P.G != 1) return pmk_synth_wide(P, io, sizeof(R) == 4 ? PM_PREC_FP32 : PM_PREC_FP64, st);
  if (P.n_pi > 1 || P.n_sig > 1) return launch_synth<R, KT, true>(P, io, st);  // a Zeeman multiplet
  return launch_synth<R, KT, false>(P, io, st);
}

}  // namespace

// Batch inversion kernels launched directly: grids wider than one warp.  Grids
// of up to 32 wavelengths are inverted by the streamed kernel (pmk_invert_stream)
// in every call path, so that each pixel's arithmetic is one compiled code.
namespace {
__global__ void fill_int_kernel(int* p, long long n, int value) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = value;
}
}  // namespace

int pmk_fill_int(int* p, int64_t n, int value, void* stream) {
  if (n <= 0) return PM_OK;
  const long long blocks = std::min<long long>((n + 255) / 256, 148 * 8);
  fill_int_kernel<<<unsigned(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(p, n, value);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "fill launch: %s", cudaGetErrorString(e)), PM_EIO;
  return PM_OK;
}

int pmk_invert(const PmParams& P, const PmIO& io, int precision, void* stream, int num_sms, float* kernel_ms) {
  if (P.G == 1) {
    snprintf(pmk_g_err, sizeof pmk_g_err, "one-warp grids are inverted by the streamed kernel");
    return PM_EINVAL;
  }
  return pmk_invert_wide(P, io, precision, stream, num_sms, kernel_ms);
}

int pmk_synth(const PmParams& P, const PmIO& io, int precision, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (P.G != 1 && P.G != 2 && P.G != 4) {
    snprintf(pmk_g_err, sizeof pmk_g_err, "nl=%d: no kernel for %d warps per pixel", P.nl, P.G);
    return PM_ERANGE;
  }
  if (precision == PM_PREC_FP32) {
    if (P.K == 9) return launch_synth_any<float, 9>(P, io, st);
    if (P.K == 10) return launch_synth_any<float, 10>(P, io, st);
    if (P.K == 11) return launch_synth_any<float, 11>(P, io, st);
  } else {
    if (P.K == 9) return launch_synth_any<double, 9>(P, io, st);
    if (P.K == 10) return launch_synth_any<double, 10>(P, io, st);
    if (P.K == 11) return launch_synth_any<double, 11>(P, io, st);
  }
  snprintf(pmk_g_err, sizeof pmk_g_err, "nterms=%d has no compiled kernel", P.K);
  return PM_ENOTSUP;
}

const char* pmk_last_cuda_error() { return pmk_g_err; }
