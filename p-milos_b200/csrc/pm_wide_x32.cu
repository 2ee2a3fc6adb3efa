// pm_wide_x32.cu -- the FP32 instances of the wide-grid kernels for Zeeman
// multiplets, macroturbulence and per-pixel wavelength grids (every combination
// but the plain one, which pm_wide.cu compiles).
#include "pm_wide_kernel.cuh"

int pmk_invert_wide_x32(const PmParams& P, const PmIO& io, void* stream, int num_sms, float* kernel_ms) {
  return invert_wide_dispatch<float, false>(P, io, static_cast<cudaStream_t>(stream), num_sms, kernel_ms);
}

int pmk_synth_wide_x32(const PmParams& P, const PmIO& io, void* stream) {
  return synth_wide_dispatch<float, false>(P, io, static_cast<cudaStream_t>(stream));
}
