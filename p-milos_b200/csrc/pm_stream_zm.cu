// pm_stream_zm.cu -- the streamed inversion kernel for Zeeman multiplets (N_PI or
// N_SIG > 1, e.g. Fe I 6301.5, 5P2.0-5D2.0): the component loop of the synthesis
// and the last component's derivative terms (ZM = true), on one grid, on a
// server's several grids, or on per-pixel grids; with a v_mac row (MAC: NTERMS
// 11, or 10 with the filling factor fixed) or without.  The launch shapes are
// those of the triplet kernels: FP32 at 4 blocks per SM (128 registers), FP64
// at 1.
#include "pm_stream_kernel.cuh"

namespace {

template <typename R, int KT, int MINB, bool MAC>
int launch_zm(const PmGridSet& GS, const PmStreamIO& sio, cudaStream_t st, int num_sms, size_t* smem_out, int wpb,
              int reserve, bool multi, bool pixgrid) {
  if (multi) return launch_invert_stream<R, KT, MINB, true, MAC, false, true>(GS, sio, st, num_sms, smem_out, wpb,
                                                                              reserve);
  if (pixgrid) return launch_invert_stream<R, KT, MINB, false, MAC, true, true>(GS, sio, st, num_sms, smem_out,
                                                                                wpb, reserve);
  return launch_invert_stream<R, KT, MINB, false, MAC, false, true>(GS, sio, st, num_sms, smem_out, wpb, reserve);
}

template <typename R, int MINB>
int launch_zm_k(const PmGridSet& GS, const PmStreamIO& sio, cudaStream_t st, int num_sms, size_t* smem_out, int wpb,
                int reserve, bool multi, bool pixgrid, int K, bool mac) {
  // NTERMS 9 never has a v_mac row and 11 always has one (milos.c:152-157)
  if (K == 9) return launch_zm<R, 9, MINB, false>(GS, sio, st, num_sms, smem_out, wpb, reserve, multi, pixgrid);
  if (K == 10 && mac)
    return launch_zm<R, 10, MINB, true>(GS, sio, st, num_sms, smem_out, wpb, reserve, multi, pixgrid);
  if (K == 10) return launch_zm<R, 10, MINB, false>(GS, sio, st, num_sms, smem_out, wpb, reserve, multi, pixgrid);
  return launch_zm<R, 11, MINB, true>(GS, sio, st, num_sms, smem_out, wpb, reserve, multi, pixgrid);
}

}  // namespace

int pmk_invert_stream_zm(const PmGridSet& GS, const PmStreamIO& sio, int precision, int warps_per_block, bool multi,
                         void* stream, int num_sms, size_t* smem_out, int reserve_blocks, bool pixgrid, bool mac) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int K = GS.g[0].K;
  if (multi && pixgrid) {
    snprintf(pmk_g_err, sizeof pmk_g_err, "pixel grids: single-grid launches only");
    return PM_EINVAL;
  }
  if (K < 9 || K > 11) {
    snprintf(pmk_g_err, sizeof pmk_g_err, "nterms=%d has no compiled kernel", K);
    return PM_ENOTSUP;
  }
  const int wpb = warps_per_block;
  if (precision == PM_PREC_FP32)
    return launch_zm_k<float, 4>(GS, sio, st, num_sms, smem_out, wpb, reserve_blocks, multi, pixgrid, K, mac);
  return launch_zm_k<double, 1>(GS, sio, st, num_sms, smem_out, wpb, reserve_blocks, multi, pixgrid, K, mac);
}
