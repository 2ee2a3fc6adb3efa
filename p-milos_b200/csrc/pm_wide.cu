// pm_wide.cu -- entry points of the kernels for wavelength grids wider than one
// warp, and their plain instances (normal triplet, no v_mac row, the grid's
// wavelengths: the benchmark workloads).  Multiplets, macroturbulence and
// per-pixel grids are compiled in pm_wide_x32.cu / pm_wide_x64.cu.
#include "pm_wide_kernel.cuh"

namespace {
bool wide_plain(const PmParams& P, const PmIO& io) {
  return P.mac_row < 0 && P.n_pi <= 1 && P.n_sig <= 1 && io.lambda_pix == nullptr;
}
}  // namespace

int pmk_invert_wide(const PmParams& P, const PmIO& io, int precision, void* stream, int num_sms, float* kernel_ms) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool f32 = precision == PM_PREC_FP32;
  if (!wide_plain(P, io))
    return f32 ? pmk_invert_wide_x32(P, io, st, num_sms, kernel_ms) : pmk_invert_wide_x64(P, io, st, num_sms, kernel_ms);
  return f32 ? invert_wide_dispatch<float, true>(P, io, st, num_sms, kernel_ms)
             : invert_wide_dispatch<double, true>(P, io, st, num_sms, kernel_ms);
}

int pmk_classical_wide(const PmParams& P, const PmIO& io, void* stream, int num_sms) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (P.G == 2) return launch_classical_wide<2>(P, io, st, num_sms);
  if (P.G == 4) return launch_classical_wide<4>(P, io, st, num_sms);
  return no_wide_kernel(P, io);
}

int pmk_synth_wide(const PmParams& P, const PmIO& io, int precision, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool f32 = precision == PM_PREC_FP32;
  const bool plain = P.mac_row < 0 && P.n_pi <= 1 && P.n_sig <= 1;
  if (!plain) return f32 ? pmk_synth_wide_x32(P, io, st) : pmk_synth_wide_x64(P, io, st);
  return f32 ? synth_wide_dispatch<float, true>(P, io, st) : synth_wide_dispatch<double, true>(P, io, st);
}
