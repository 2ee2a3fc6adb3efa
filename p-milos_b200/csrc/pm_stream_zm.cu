// pm_stream_zm.cu -- the streamed inversion kernel for Zeeman multiplets (N_PI or
// N_SIG > 1, e.g. Fe I 6301.5, 5P2.0-5D2.0): the component loop of the synthesis
// and the last component's derivative terms (ZM = true), on one grid, on a
// server's several grids, or on per-pixel grids.  Multiplets carry no
// macroturbulence row, so NTERMS is 9 or 10 (the filling factor).  The launch
// shapes are those of the triplet kernels: FP32 at 4 blocks per SM (128
// registers), FP64 at 1.
#include "pm_stream_kernel.cuh"

namespace {

template <typename R, int KT, int MINB>
int launch_zm(const PmGridSet& GS, const PmStreamIO& sio, cudaStream_t st, int num_sms, size_t* smem_out, int wpb,
              int reserve, bool multi, bool pixgrid) {
  if (multi) return launch_invert_stream<R, KT, MINB, true, false, false, true>(GS, sio, st, num_sms, smem_out, wpb,
                                                                                reserve);
  if (pixgrid) return launch_invert_stream<R, KT, MINB, false, false, true, true>(GS, sio, st, num_sms, smem_out,
                                                                                  wpb, reserve);
  return launch_invert_stream<R, KT, MINB, false, false, false, true>(GS, sio, st, num_sms, smem_out, wpb, reserve);
}

}  // namespace

int pmk_invert_stream_zm(const PmGridSet& GS, const PmStreamIO& sio, int precision, int warps_per_block, bool multi,
                         void* stream, int num_sms, size_t* smem_out, int reserve_blocks, bool pixgrid) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int K = GS.g[0].K;
  if (multi && pixgrid) {
    snprintf(pmk_g_err, sizeof pmk_g_err, "pixel grids: single-grid launches only");
    return PM_EINVAL;
  }
  if (K != 9 && K != 10) {
    snprintf(pmk_g_err, sizeof pmk_g_err, "Zeeman multiplets: nterms=%d (9 or 10 without macroturbulence)", K);
    return PM_ENOTSUP;
  }
  const int wpb = warps_per_block;
  if (precision == PM_PREC_FP32)
    return K == 9 ? launch_zm<float, 9, 4>(GS, sio, st, num_sms, smem_out, wpb, reserve_blocks, multi, pixgrid)
                  : launch_zm<float, 10, 4>(GS, sio, st, num_sms, smem_out, wpb, reserve_blocks, multi, pixgrid);
  return K == 9 ? launch_zm<double, 9, 1>(GS, sio, st, num_sms, smem_out, wpb, reserve_blocks, multi, pixgrid)
                : launch_zm<double, 10, 1>(GS, sio, st, num_sms, smem_out, wpb, reserve_blocks, multi, pixgrid);
}
