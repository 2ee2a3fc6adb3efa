// pm_wide_kernel.cuh -- kernels for wavelength grids wider than one warp (32 <
// nl <= 128: two or four warps per pixel, thread t = wavelength t), their
// launchers and the dispatch over compiled instances.  Internal header of the
// translation units that instantiate them: pm_wide.cu (the plain instances:
// normal triplet, no v_mac row, the grid's wavelengths), pm_wide_x32.cu and
// pm_wide_x64.cu (every other combination, FP32 and FP64).  Everything here has
// internal linkage.
#pragma once
#include "pm_device.cuh"

namespace {
// ---------------------------------------------------------------------------
// Wide grids: 32 < nl <= 128.  G = 2 or 4 warps invert one pixel; the block is
// one pixel group and thread t owns wavelength t.  The per-wavelength work
// (synthesis, response functions, their terms of chi^2 and of the normal
// equations) is the one-warp code; what crosses warps goes through shared
// memory: the PSF correlations read neighbouring wavelengths' rows, sums are
// reduced per warp by shuffles and then across the G warps in a fixed order (so
// every thread holds the same total), and warp 0 alone runs the damped solve.
// ---------------------------------------------------------------------------
template <typename R, int G>
struct alignas(16) WideSmem {
  static constexpr int NT = 32 * G;                 // threads = wavelength slots
  static constexpr int VEC = 16 / sizeof(R);
  static constexpr int RS = 32 + VEC;               // RF row stride: conflict-free 16-byte row reads
  static constexpr int RED = 96;                    // reduction slots per warp
  R xs[NT][4];                 // synthesized (I, Q, U, V) per wavelength: the PSF input
  R rf[NT][RS];                // response functions [lambda][profile]; solver scratch
  R ls[NT][kLaneStatePad];     // synthesis state per wavelength
  ModelTerms<R> mt;
  SolveSmem sv;
  double red[2][G][RED];       // per-warp partial sums, double-buffered
  double model[11], trial[11];
  // the shared stray-light profile [4][nl] (PM_SLIGHT_SHARED): thread-indexed
  // reads of the parameter block would be serialised by the constant cache
  float sl[4 * NT];
  unsigned long long pix;
};

// The block's copy of the shared stray-light profile (every thread calls it; the
// caller's next barrier publishes it) and the profile a pixel mixes in.
template <typename R, int G>
__device__ __forceinline__ void load_slight_wide(const PmParams& P, WideSmem<R, G>& sm) {
  if (P.slight_mode == PM_SLIGHT_SHARED)
    for (int e = threadIdx.x; e < 4 * WideSmem<R, G>::NT; e += 32 * G) sm.sl[e] = e < 4 * P.nl ? P.sl_f[e] : 0.0f;
}
template <typename R, int G>
__device__ __forceinline__ const float* slight_of_wide(const PmParams& P, const WideSmem<R, G>& sm,
                                                       const float* cube, size_t base) {
  if (P.slight_mode == PM_SLIGHT_SHARED) return sm.sl;
  if (P.slight_mode == PM_SLIGHT_PER_PIXEL && cube) return cube + base;
  return nullptr;
}

template <typename R, int G>
constexpr bool wide_layout_ok() {
  using W = WideSmem<R, G>;
  return offsetof(W, xs) % 16 == 0 && offsetof(W, rf) % 16 == 0 && offsetof(W, ls) % 16 == 0 &&
         offsetof(W, mt) % 16 == 0 && (W::RS * sizeof(R)) % 16 == 0 && (4 * sizeof(R)) % 16 == 0 &&
         sizeof(W::rf) >= eigen_scratch_doubles<11>() * sizeof(double) && sizeof(W) % 16 == 0;
}
static_assert(wide_layout_ok<float, 2>() && wide_layout_ok<float, 4>(), "wide shared-memory layout (float)");
static_assert(wide_layout_ok<double, 2>() && wide_layout_ok<double, 4>(), "wide shared-memory layout (double)");

// Sum N values over the block: per warp by shuffles, then the G warp totals in
// warp order from red[slot] ([2][G][STRIDE]).  Every thread returns the same
// totals.  The slot alternates between calls, so one barrier per call suffices:
// a slot is rewritten only after the next call's barrier, which every thread
// reaches after reading this call's totals.
template <int G, int STRIDE, int N>
__device__ __forceinline__ void block_sum(double* red, int& slot, double (&v)[N]) {
  static_assert(N <= STRIDE, "too many sums for the reduction slots");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = warp_sum(v[i]);
  double* r = red + slot * G * STRIDE;
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < N; ++i) r[warp * STRIDE + i] = v[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < N; ++i) {
    double t = r[i];
#pragma unroll
    for (int g = 1; g < G; ++g) t += r[g * STRIDE + i];
    v[i] = t;
  }
  slot ^= 1;
}

template <typename R>
__device__ __forceinline__ void store4(R* dst, const R S[4]) {
  if constexpr (sizeof(R) == 4) {
    *reinterpret_cast<float4*>(dst) = make_float4(S[0], S[1], S[2], S[3]);
  } else {
    reinterpret_cast<double2*>(dst)[0] = make_double2(S[0], S[1]);
    reinterpret_cast<double2*>(dst)[1] = make_double2(S[2], S[3]);
  }
}

template <typename R>
__device__ __forceinline__ void load4(const R* src, R x[4]) {
  if constexpr (sizeof(R) == 4) {
    const float4 q = *reinterpret_cast<const float4*>(src);
    x[0] = q.x; x[1] = q.y; x[2] = q.z; x[3] = q.w;
  } else {
    const double2 a = reinterpret_cast<const double2*>(src)[0], b = reinterpret_cast<const double2*>(src)[1];
    x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y;
  }
}

// PSF correlation of the four synthesized profiles across the block (the
// convolution psf_rows does within a warp): thread t forms output t from the
// rows t + j - nl/2 of the in-grid taps j in [tap_lo, tap_hi].  Stokes I is
// Ic (1 - W_t) + sum_j G_j I_{t+j-nl/2}, which equals Ic - sum_j G_j (Ic - I).
// The caller separates the reads here from the next call's writes by a barrier.
template <typename R, int G>
__device__ __forceinline__ void psf_wide(const PmParams& P, WideSmem<R, G>& sm, int t, bool valid, R omw_t,
                                         R S[4]) {
  if (valid) store4<R>(sm.xs[t], S);
  __syncthreads();
  const int nl = P.nl;
  const R i0 = sm.xs[0][0], in = sm.xs[nl - 1][0];
  const R ic = (i0 > in) ? i0 : in;
  R acc[4] = {R(0), R(0), R(0), R(0)};
  const int b = t - P.half;
#pragma unroll 2
  for (int j = P.tap_lo; j <= P.tap_hi; ++j) {
    const int mm = b + j;
    if (mm >= 0 && mm < nl) {
      const R g = taps<R>(P, j);
      R x[4];
      load4<R>(sm.xs[mm], x);
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma(g, x[q], acc[q]);
    }
  }
  S[0] = valid ? fma(ic, omw_t, acc[0]) : R(0);
#pragma unroll
  for (int q = 1; q < 4; ++q) S[q] = valid ? acc[q] : R(0);
}

// ---------------------------------------------------------------------------
// Macroturbulence on a wide grid (the direct branch of mil_sinrf.c:288-357 and
// me_der.c:314-438, as the one-warp mac_* helpers do it): thread t builds the
// Gaussian's value at wavelength t, the block normalises it to unit sum (summed
// in wavelength order, as fgauss does), correlates it with the PSF when there
// is one (direct_convolution_double, all nl taps, FP64), and the profiles,
// every response function but S0's and the v_mac row are circular convolutions
// with it, rotated by nl/2 as convCircular returns them.  The data live in
// dynamic shared memory after WideSmem, in the macroturbulence instances only.
// ---------------------------------------------------------------------------
template <typename R, int G>
struct alignas(16) MacSmem {
  static constexpr int NT = 32 * G;
  double s[2][NT];  // the Gaussian (and its derivative) in FP64 while they are built
  R k[3 * NT];      // the kernel, tripled: k[u] = kernel[u mod nl] for u < 3 nl
  R kd[3 * NT];     // the same for the derivative in v_mac
};

template <typename R, int G>
__device__ __forceinline__ MacSmem<R, G>& mac_smem(WideSmem<R, G>& sm) {
  return *reinterpret_cast<MacSmem<R, G>*>(reinterpret_cast<unsigned char*>(&sm) + sizeof(WideSmem<R, G>));
}

// The kernel of v_mac (and with DERIV its derivative, in the form of
// me_der.c:419-421) into MacSmem::k (kd).  Every thread of the block calls it;
// the caller puts a barrier between it and the reads of k / kd.  dl_t: the
// offset lambda - lambda0 of wavelength t; lp: the pixel's own wavelengths, or
// nullptr for the grid's.
template <typename R, int G, bool DERIV>
__device__ __forceinline__ void mac_kernel_wide(const PmParams& P, WideSmem<R, G>& sm, double mac, int t, bool valid,
                                                double dl_t, const double* lp) {
  MacSmem<R, G>& mx = mac_smem(sm);
  const int nl = P.nl;
  const double dl_c = lp ? lp[P.half] - P.lambda0 : P.dl[P.half];
  const double x = valid ? dl_t - dl_c : 0.0;  // lambda_t - lambda[nl/2], exactly
  const double ild = (P.lambda0 * mac) / kVLight;
  const double a = x / ild;
  const double term = (a * a) / 2;
  double g = (valid && term < 1e30) ? exp(-term) : 0.0;
  mx.s[0][t] = g;
  __syncthreads();
  double sum = 0.0;
  for (int u = 0; u < nl; ++u) sum += mx.s[0][u];
  g = g / sum;
  double gd = DERIV ? g / mac * (a * a - 1.0) : 0.0;
  if (P.has_psf) {
    __syncthreads();  // every thread has its sum
    mx.s[0][t] = g;
    if (DERIV) mx.s[1][t] = gd;
    __syncthreads();
    double acc = 0.0, accd = 0.0;
    for (int j = 0; j < nl; ++j) {
      const int u = t + j - P.half;
      if (u >= 0 && u < nl) {
        acc = fma(P.taps_d[j], mx.s[0][u], acc);
        if (DERIV) accd = fma(P.taps_d[j], mx.s[1][u], accd);
      }
    }
    g = acc;
    gd = accd;
  }
  if (valid) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      mx.k[t + q * nl] = R(g);
      if (DERIV) mx.kd[t + q * nl] = R(gd);
    }
  }
}

// out[s] at wavelength t: sum_u xs[u][s] k3[(t + nl/2 - u) mod nl] over the
// unconvolved synthesis in xs; k3 is a tripled kernel of MacSmem.
template <typename R, int G>
__device__ __forceinline__ void mac_circular_wide(const PmParams& P, const WideSmem<R, G>& sm, const R* k3, int t,
                                                  bool valid, R out[4]) {
  R acc[4] = {R(0), R(0), R(0), R(0)};
  const R* kb = k3 + (valid ? t : 0) + P.half + P.nl;
#pragma unroll 2
  for (int u = 0; u < P.nl; ++u) {
    const R kk = kb[-u];
    R x[4];
    load4<R>(sm.xs[u], x);
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = fma(x[q], kk, acc[q]);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) out[q] = valid ? acc[q] : R(0);
}

// The 32 response-function profiles of the rows sm.rf[u] convolved circularly
// with the kernel, at wavelength t.
template <typename R, int G>
__device__ __forceinline__ void mac_rf_wide(const PmParams& P, WideSmem<R, G>& sm, int t, bool valid, R (&v)[32]) {
  constexpr int VEC = WideSmem<R, G>::VEC;
#pragma unroll
  for (int p = 0; p < 32; ++p) v[p] = 0;
  const R* kb = mac_smem(sm).k + (valid ? t : 0) + P.half + P.nl;
#pragma unroll 1
  for (int u = 0; u < P.nl; ++u) {
    const R g = kb[-u];
    const R* row = sm.rf[u];
#pragma unroll
    for (int p = 0; p < 32; p += VEC) {
      if constexpr (VEC == 4) {
        const float4 q = *reinterpret_cast<const float4*>(row + p);
        v[p] = fma(q.x, g, v[p]);
        v[p + 1] = fma(q.y, g, v[p + 1]);
        v[p + 2] = fma(q.z, g, v[p + 2]);
        v[p + 3] = fma(q.w, g, v[p + 3]);
      } else {
        const double2 q = *reinterpret_cast<const double2*>(row + p);
        v[p] = fma(q.x, g, v[p]);
        v[p + 1] = fma(q.y, g, v[p + 1]);
      }
    }
  }
}

// MAC: compiled with the macroturbulence branch (the grid has a v_mac row).
// dl_t: the offset lambda - lambda0 of wavelength t; lp: the pixel's own
// wavelengths, or nullptr for the grid's.
template <typename R, int G, bool ZM, bool MAC>
__device__ __forceinline__ void synthesize_wide(const PmParams& P, WideSmem<R, G>& sm, const double* m,
                                                const float* sl_pix, int t, bool valid, double dl_t, const double* lp,
                                                R omw_t, R S[4], R Su[4]) {
  ModelTerms<R> T;
  LaneState<R> st;
  model_terms<R, ZM>(P, m, T);
  synth_lane<R, ZM>(P, T, dl_t, st, S);
  copy16(*reinterpret_cast<LaneState<R>*>(sm.ls[t]), st);
  if (t == 0) copy16(sm.mt, T);
  const double mac = MAC ? m[9] : 0.0;
  if (MAC && mac > kMacMin) {
    // every profile (Stokes I with no continuum padding) convolved circularly;
    // xs keeps the unconvolved synthesis for the v_mac row
    if (valid) store4<R>(sm.xs[t], S);
    mac_kernel_wide<R, G, false>(P, sm, mac, t, valid, dl_t, lp);
    __syncthreads();
    mac_circular_wide<R, G>(P, sm, mac_smem(sm).k, t, valid, S);
  } else if (P.has_psf) {
    psf_wide<R, G>(P, sm, t, valid, omw_t, S);
  }
#pragma unroll
  for (int s = 0; s < 4; ++s) Su[s] = S[s];
  if (P.slight_mode != PM_SLIGHT_NONE) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int idx = s * P.nl + (valid ? t : 0);
      const R slv = R(sl_pix[idx]);  // shared profile (block copy) or the pixel's own
      S[s] = S[s] * T.alf + slv * T.oma;
    }
  }
}

// PSF correlation of the 32 response-function profiles across the block: thread
// t forms output t of every profile from rows t + j - nl/2 (eight 16-byte loads
// and 32 FMAs per tap).  Stokes-I profiles add Ic (1 - W_t), Ic = max of the
// profile's end points (me_der.c:471-496).
template <typename R, int G>
__device__ __forceinline__ void rf_correlate_wide(const PmParams& P, const WideSmem<R, G>& sm, int t, R omw_t,
                                                  R (&v)[32]) {
  constexpr int VEC = WideSmem<R, G>::VEC;
  const int nl = P.nl;
#pragma unroll
  for (int p = 0; p < 32; ++p) v[p] = 0;
  const int b = t - P.half;
#pragma unroll 1
  for (int j = P.tap_lo; j <= P.tap_hi; ++j) {
    const int mm = b + j;
    if (mm >= 0 && mm < nl) {
      const R g = taps<R>(P, j);
      const R* row = sm.rf[mm];
#pragma unroll
      for (int p = 0; p < 32; p += VEC) {
        if constexpr (VEC == 4) {
          const float4 q = *reinterpret_cast<const float4*>(row + p);
          v[p] = fma(g, q.x, v[p]);
          v[p + 1] = fma(g, q.y, v[p + 1]);
          v[p + 2] = fma(g, q.z, v[p + 2]);
          v[p + 3] = fma(g, q.w, v[p + 3]);
        } else {
          const double2 q = *reinterpret_cast<const double2*>(row + p);
          v[p] = fma(g, q.x, v[p]);
          v[p + 1] = fma(g, q.y, v[p + 1]);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const R e0 = sm.rf[0][4 * r], en = sm.rf[nl - 1][4 * r];
    v[4 * r] = fma((e0 > en) ? e0 : en, omw_t, v[4 * r]);
  }
}

// Response functions of the last synthesis at this thread's wavelength, after
// correlation, stray light and filling factor (as gather_rf): d[row][stokes].
// Sff is the spectrum the filling-factor row is built from.
// mac: v_mac of the model of the last synthesis (MAC instances); dl_t, lp: as
// for synthesize_wide.
template <typename R, int KT, int G, bool ZM, bool MAC>
__device__ __forceinline__ void rf_wide(const PmParams& P, WideSmem<R, G>& sm, int t, bool valid, R omw_t,
                                        const R Sff[4], const float* sl_pix, double mac, double dl_t,
                                        const double* lp, R (&d)[KT][4]) {
  const bool mac_on = MAC && mac > kMacMin;
  if (mac_on) mac_kernel_wide<R, G, true>(P, sm, mac, t, valid, dl_t, lp);
  R alf;
  {
    ModelTerms<R> T;
    copy16(T, sm.mt);
    LaneState<R> st;
    copy16(st, *reinterpret_cast<const LaneState<R>*>(sm.ls[t]));
    rf_lane<R, 1, ZM>(P, T, st, sm.rf[t], valid);
    alf = T.alf;
  }
  __syncthreads();
  R v[32];
  R dmac[4] = {R(0), R(0), R(0), R(0)};
  if (mac_on) {
    mac_rf_wide<R, G>(P, sm, t, valid, v);
    mac_circular_wide<R, G>(P, sm, mac_smem(sm).kd, t, valid, dmac);
  } else if (P.has_psf) {
    rf_correlate_wide<R, G>(P, sm, t, omw_t, v);
  } else {
#pragma unroll
    for (int p = 0; p < 32; ++p) v[p] = sm.rf[t][p];
  }
#pragma unroll
  for (int r = 0; r < KT; ++r) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      R x;
      if (r < 7) x = v[r * 4 + s];
      else if (r == 7) x = (s == 0) ? R(1) : R(0);  // S0 (me_der.c:301-306)
      else if (r == 8) x = v[7 * 4 + s];
      else if (MAC && r == 9 && P.mac_row == 9) x = dmac[s];  // zero while v_mac <= 1e-4
      else x = R(0);
      d[r][s] = valid ? x : R(0);
    }
  }
  if (P.slight_mode != PM_SLIGHT_NONE) {
#pragma unroll
    for (int r = 0; r < KT; ++r) {
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        d[r][s] = d[r][s] * alf;
        if (r == P.ff_row) {
          const int idx = s * P.nl + (valid ? t : 0);
          const R slv = R(sl_pix[idx]);
          d[r][s] = valid ? Sff[s] - slv : R(0);
        }
      }
    }
  }
}

// Normal equations over the block: packed entries reduced per warp (as
// normal_eq), then the G warp totals summed in warp order into sv.ab.
template <typename R, int KT, int G>
__device__ __forceinline__ void normal_eq_wide(const PmParams& P, WideSmem<R, G>& sm, int& slot,
                                               const R (&d)[KT][4], const R S[4], const float O[4],
                                               const R isig[4]) {
  constexpr int NA = KT * (KT + 1) / 2;
  constexpr int NT = NA + KT;
  constexpr int NCH = (NT + 31) / 32;
  constexpr int RED = WideSmem<R, G>::RED;
  static_assert(NCH * 32 <= RED, "reduction slots too small");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  R cw[4], rw[4];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    cw[s] = R(P.w[s]) * isig[s];
    rw[s] = R(P.w[s]) * (S[s] - R(O[s])) * isig[s];
  }
  double* red = &sm.red[slot][0][0];
  double* mine = red + warp * RED;
  ne_reduce_chunk<R, KT, 0>(mine, lane, d, cw, rw);
  if constexpr (NCH > 1) ne_reduce_chunk<R, KT, 1>(mine, lane, d, cw, rw);
  if constexpr (NCH > 2) ne_reduce_chunk<R, KT, 2>(mine, lane, d, cw, rw);
  __syncthreads();
  for (int e = threadIdx.x; e < KT * KT + KT; e += 32 * G) {
    int idx;
    if (e < KT * KT) {
      int a = e / KT, b = e % KT;
      if (a > b) { int tt = a; a = b; b = tt; }
      idx = a * KT - (a * (a - 1)) / 2 + (b - a);
    } else {
      idx = NA + (e - KT * KT);
    }
    double val = red[idx];
#pragma unroll
    for (int g = 1; g < G; ++g) val += red[g * RED + idx];
    sm.sv.ab[e] = val;
  }
  slot ^= 1;
  __syncthreads();
}

template <typename R, int G>
__device__ __forceinline__ double chisq_wide(const PmParams& P, WideSmem<R, G>& sm, int& slot, const R S[4],
                                             const float O[4], const R isig[4], bool valid, double nfree) {
  double acc[1] = {0.0};
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const R dif = S[s] - R(O[s]);
    acc[0] += valid ? double(dif * dif) * P.w[s] * double(isig[s]) : 0.0;
  }
  block_sum<G, WideSmem<R, G>::RED>(&sm.red[0][0][0], slot, acc);
  return acc[0] / nfree;
}

template <typename R, int KT, int G, bool ZM, bool MAC>
__device__ __forceinline__ void rf_and_normal_eq_wide(const PmParams& P, WideSmem<R, G>& sm, int& slot, int t,
                                                      bool valid, R omw_t, const R S[4], const R Sff[4],
                                                      const float O[4], const R isig[4], const float* sl_pix,
                                                      double mac, double dl_t, const double* lp) {
  R d[KT][4];
  rf_wide<R, KT, G, ZM, MAC>(P, sm, t, valid, omw_t, Sff, sl_pix, mac, dl_t, lp, d);
#pragma unroll
  for (int r = 0; r < KT; ++r)
    if (P.zero_row[r]) {
#pragma unroll
      for (int s = 0; s < 4; ++s) d[r][s] = 0;
    }
  normal_eq_wide<R, KT, G>(P, sm, slot, d, S, O, isig);
}

// lm_mils over pixels of a wide grid: the control flow of invert_pixel with
// block-wide reductions; the solve and the trial model come from warp 0.
// ZM: the line is a Zeeman multiplet (a separate instance, as in the one-warp
// kernel); MAC: the grid has a v_mac row (dynamic shared memory holds MacSmem);
// PIXGRID: every pixel has its own wavelengths (io.lambda_pix).
template <typename R, int KT, int G, int MINB, bool ZM, bool MAC, bool PIXGRID>
__global__ void __launch_bounds__(32 * G, MINB) invert_wide_kernel(const __grid_constant__ PmParams P,
                                                                     const PmIO io) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WideSmem<R, G>& sm = *reinterpret_cast<WideSmem<R, G>*>(smem_raw);
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const bool valid = t < P.nl;
  double dl_t = P.dl[valid ? t : 0];
  const R omw_t = valid ? omw<R>(P, t) : R(0);
  double* m = sm.model;
  double* trial = sm.trial;
  int slot = 0;
  load_slight_wide<R, G>(P, sm);  // published by the loop's first barrier

  while (true) {
    if (t == 0) sm.pix = atomicAdd(&io.ctr[PMC_NEXT], 1ull);
    __syncthreads();
    const unsigned long long pix = sm.pix;
    if (pix >= (unsigned long long)io.npix) break;
    // the pixel's own wavelengths (the PSF taps stay the context's)
    const double* lp = PIXGRID ? io.lambda_pix + size_t(pix) * P.nl : nullptr;
    if constexpr (PIXGRID) dl_t = lp[valid ? t : 0] - P.lambda0;
    const size_t base = size_t(pix) * 4 * P.nl;
    const float* sl_pix = slight_of_wide<R, G>(P, sm, io.slight, base);

    float O[4];
    R isig[4];
    double gh[1] = {0.0};
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      O[s] = valid ? io.spectro[base + s * P.nl + t] : 0.0f;
      const bool g = valid && O[s] <= -1.0f;
      gh[0] += g ? 1.0 : 0.0;
      isig[s] = R(1.0 / (g ? kGhostSigma : P.noise));
    }
    if (t < 11) m[t] = P.classical ? io.models_out[size_t(pix) * 11 + t] : P.guess[t];
    block_sum<G, WideSmem<R, G>::RED>(&sm.red[0][0][0], slot, gh);  // also publishes m

    const int nfree = P.nfree_base - int(gh[0]);
    int status = PM_PIX_MAXITER, iter = 0, accepted = 0, fallbacks = 0;
    double ochi = 0;
    R S[4];
    if (nfree == 0) {
      status = PM_PIX_NFREE;
      iter = -1;
#pragma unroll
      for (int s = 0; s < 4; ++s) S[s] = 0;
    } else {
      // the starting model's synthesis and response functions run as the
      // loop's first pass (accepted without a step), so that each is inlined
      // once; lm_mils' order of operations is unchanged
      double chi0 = 0, flambda = P.ilambda, factor = 1.0;
      if (t < 11) trial[t] = m[t];
      __syncthreads();
      bool stop = false, first = true;
      while (true) {
        if (!first) {
          if (warp == 0) {
            double dlt[KT];
            bool ok = true;
            double* scratch = reinterpret_cast<double*>(&sm.rf[0][0]);  // idle during the solve
            if (P.solver == PM_SOLVE_CHOLESKY) ok = solve_cholesky<KT>(sm.sv, scratch, lane, flambda, dlt);
            if (P.solver != PM_SOLVE_CHOLESKY || !ok) {
              if (P.solver == PM_SOLVE_CHOLESKY) ++fallbacks;
              solve_eigen<KT>(sm.sv, scratch, lane, flambda);
#pragma unroll
              for (int i = 0; i < KT; ++i) dlt[i] = sm.sv.delta[i];
              __syncwarp();
            }
            double tt[11];
#pragma unroll
            for (int i = 0; i < 11; ++i) tt[i] = trial[i];
            apply_delta<KT>(P, m, dlt, tt);
            check_model(tt);
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 11; ++i)
              if (lane == i) trial[i] = tt[i];
          }
          __syncthreads();
        }
        R Su[4];
        synthesize_wide<R, G, ZM, MAC>(P, sm, trial, sl_pix, t, valid, dl_t, lp, omw_t, S, Su);
        const double chi = chisq_wide<R, G>(P, sm, slot, S, O, isig, valid, double(nfree));
        bool accept = true;
        if (!first) {
          if ((fabs((ochi - chi) * 100 / chi) < P.toplim) || (chi < 0.0001)) {
            stop = true;
            status = PM_PIX_CONVERGED;
          }
          accept = chi - ochi < 0.;
        }
        if (accept) {
          if (!first) flambda = flambda / (5.0 * factor);
          if (t < 11) m[t] = trial[t];
          // the filling-factor row: unmixed synthesis first, mixed after a step
          // (milosUtils.c:537 vs :587)
          R Sff[4];
#pragma unroll
          for (int s = 0; s < 4; ++s) Sff[s] = first ? Su[s] : S[s];
          rf_and_normal_eq_wide<R, KT, G, ZM, MAC>(P, sm, slot, t, valid, omw_t, S, Sff, O, isig, sl_pix,
                                                   MAC ? trial[9] : 0.0, dl_t, lp);
          ochi = chi;
          if (first) chi0 = chi;
          else ++accepted;
        } else {
          flambda = flambda * 10.0 * factor;
        }
        if (!first) {
          if ((flambda > 1e+7) || (flambda < 1e-25)) {
            if (!stop) status = PM_PIX_LAMBDA;
            stop = true;
          }
          ++iter;
          if (P.logclambda) factor = double(log10f(float(chi)) / log10f(float(chi0)));
          if (!(iter < P.miter && !stop)) break;  // lm_mils' do-while: at least one step
        }
        first = false;
      }
      __syncthreads();  // the last accepted model in m is visible to every thread
      bool finite = isfinite(ochi);
#pragma unroll
      for (int i = 0; i < 11; ++i) finite = finite && isfinite(m[i]);
      if (!finite) status = PM_PIX_NONFINITE;
    }
    if (t < 11) io.models_out[size_t(pix) * 11 + t] = m[t];
    if (t == 0) {
      io.chisq_out[pix] = float(ochi);
      io.iters_out[pix] = iter;
      if (io.status_out) io.status_out[pix] = status;
      atomicAdd(&io.ctr[PMC_ITERS], (unsigned long long)(iter > 0 ? iter : 0));
      atomicAdd(&io.ctr[PMC_ACCEPTED], (unsigned long long)accepted);
      if (fallbacks) atomicAdd(&io.ctr[PMC_FALLBACK], (unsigned long long)fallbacks);
    }
    if (io.spectra_out && valid) {
#pragma unroll
      for (int s = 0; s < 4; ++s) io.spectra_out[base + s * P.nl + t] = float(S[s]);
    }
    __syncthreads();
  }
}

// Classical estimates for wide grids, one block of G warps per pixel.
template <int G>
__global__ void __launch_bounds__(32 * G) classical_wide_kernel(const __grid_constant__ PmParams P, const PmIO io) {
  constexpr int STR = 16;
  __shared__ double red[2 * G * STR];
  __shared__ unsigned mask[2][G];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const bool valid = t < P.nl;
  int slot = 0, ms = 0;
  for (int64_t pix = blockIdx.x; pix < io.npix; pix += gridDim.x) {
    const size_t base = size_t(pix) * 4 * P.nl;
    float O[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) O[s] = valid ? io.spectro[base + s * P.nl + t] : 0.0f;
    const unsigned nn = __ballot_sync(kFull, valid && !(O[0] < 0.0f));
    if (lane == 0) mask[ms][warp] = nn;
    __syncthreads();
    // leading and trailing ghost wavelengths (I < 0)
    int begin = -1, end = -1;
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const unsigned k = mask[ms][g];
      if (k) {
        if (begin < 0) begin = 32 * g + __ffs(k) - 1;
        end = 32 * g + 32 - __clz(k);
      }
    }
    ms ^= 1;
    // every intensity negative (begin < 0, uniform over the block): no estimate, the guess stays
    double v[10];
    if (begin >= 0) {
      const double Ic = double(io.spectro[base + end - 1]);
      const int tt = valid ? t : 0;
      const double dl = io.lambda_pix ? io.lambda_pix[size_t(pix) * P.nl + tt] - P.lambda0 : P.dl[tt];
      classical_terms(P, O, t, dl, valid, begin, end, Ic, v);
      block_sum<G, STR>(red, slot, v);
    }
    if (t < 11) {
      double g[11];
#pragma unroll
      for (int i = 0; i < 11; ++i) g[i] = P.guess[i];
      if (begin >= 0) classical_finish<true>(P, v, g);
      double out = g[0];
#pragma unroll
      for (int i = 1; i < 11; ++i)
        if (t == i) out = g[i];
      io.models_out[size_t(pix) * 11 + t] = out;
    }
  }
}

// Synthesis (and response functions) of given models on a wide grid.
template <typename R, int KT, int G, bool ZM, bool MAC>
__global__ void __launch_bounds__(32 * G) synth_wide_kernel(const __grid_constant__ PmParams P, const PmIO io) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WideSmem<R, G>& sm = *reinterpret_cast<WideSmem<R, G>*>(smem_raw);
  const int t = threadIdx.x;
  const bool valid = t < P.nl;
  double dl_t = P.dl[valid ? t : 0];
  const R omw_t = valid ? omw<R>(P, t) : R(0);
  load_slight_wide<R, G>(P, sm);  // published by the loop's first barrier
  for (int64_t pix = blockIdx.x; pix < io.npix; pix += gridDim.x) {
    const size_t base = size_t(pix) * 4 * P.nl;
    const float* sl_pix = slight_of_wide<R, G>(P, sm, io.slight, base);
    const double* lp = io.lambda_pix ? io.lambda_pix + size_t(pix) * P.nl : nullptr;  // the pixel's own wavelengths
    if (lp) dl_t = lp[valid ? t : 0] - P.lambda0;
    if (t < 11) sm.model[t] = io.models_in[size_t(pix) * 11 + t];
    __syncthreads();
    R S[4], Su[4];
    synthesize_wide<R, G, ZM, MAC>(P, sm, sm.model, sl_pix, t, valid, dl_t, lp, omw_t, S, Su);
    if (valid) {
#pragma unroll
      for (int s = 0; s < 4; ++s) io.spectra_out[base + s * P.nl + t] = float(S[s]);
    }
    if (io.rf_out) {
      __syncthreads();  // the model terms from thread 0
      R d[KT][4];
      rf_wide<R, KT, G, ZM, MAC>(P, sm, t, valid, omw_t, Su, sl_pix, MAC ? sm.model[9] : 0.0, dl_t, lp, d);
      if (valid) {
        const size_t rb = size_t(pix) * 4 * KT * P.nl;
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
          for (int r = 0; r < KT; ++r) io.rf_out[rb + (size_t(s) * KT + r) * P.nl + t] = float(d[r][s]);
      }
    }
    __syncthreads();
  }
}


using WideKernel = void (*)(const PmParams, const PmIO);

// The classical estimates of every pixel into io.models_out, one block of G
// warps per pixel, up to 64 / G blocks per SM.
template <int G>
int launch_classical_wide(const PmParams& P, const PmIO& io, cudaStream_t st, int num_sms) {
  int64_t cb = io.npix;
  if (cb > int64_t(num_sms) * (64 / G)) cb = int64_t(num_sms) * (64 / G);
  if (cb < 1) cb = 1;
  classical_wide_kernel<G><<<unsigned(cb), 32 * G, 0, st>>>(P, io);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "classical launch: %s", cudaGetErrorString(e)), PM_EIO;
  return PM_OK;
}

// One compiled instance of the wide inversion: the classical estimates first
// when the settings ask for them, then the LM kernel with as many blocks as fit.
template <typename R, int KT, int G, int MINB, bool ZM, bool MAC, bool PIXGRID>
int launch_invert_wide_inst(const PmParams& P, const PmIO& io, cudaStream_t st, int num_sms, float* kernel_ms) {
  const int threads = 32 * G;
  const size_t smem = sizeof(WideSmem<R, G>) + (MAC ? sizeof(MacSmem<R, G>) : 0);
  const WideKernel kern = invert_wide_kernel<R, KT, G, MINB, ZM, MAC, PIXGRID>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "%s", cudaGetErrorString(e)), PM_EIO;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (e != cudaSuccess || per_sm < 1) return snprintf(pmk_g_err, sizeof pmk_g_err, "occupancy: %s", cudaGetErrorString(e)), PM_EIO;
  int64_t blocks = int64_t(per_sm) * num_sms;
  if (blocks > io.npix) blocks = io.npix > 0 ? io.npix : 1;
  cudaEvent_t a = nullptr, b = nullptr;
  if (kernel_ms) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, st);
  }
  int rc = PM_OK;
  if (P.classical) rc = launch_classical_wide<G>(P, io, st, num_sms);
  if (rc == PM_OK) {
    kern<<<unsigned(blocks), threads, smem, st>>>(P, io);
    e = cudaGetLastError();
  }
  if (kernel_ms) {
    if (rc == PM_OK) {
      cudaEventRecord(b, st);
      cudaEventSynchronize(b);
      cudaEventElapsedTime(kernel_ms, a, b);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  if (rc != PM_OK) return rc;
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "invert launch: %s", cudaGetErrorString(e)), PM_EIO;
  return PM_OK;
}

template <typename R, int KT, int G, bool ZM, bool MAC>
int launch_synth_wide_inst(const PmParams& P, const PmIO& io, cudaStream_t st) {
  const int threads = 32 * G;
  const size_t smem = sizeof(WideSmem<R, G>) + (MAC ? sizeof(MacSmem<R, G>) : 0);
  const WideKernel kern = synth_wide_kernel<R, KT, G, ZM, MAC>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "%s", cudaGetErrorString(e)), PM_EIO;
  int64_t blocks = io.npix;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  kern<<<unsigned(blocks), threads, smem, st>>>(P, io);
  e = cudaGetLastError();
  if (e != cudaSuccess) return snprintf(pmk_g_err, sizeof pmk_g_err, "synth launch: %s", cudaGetErrorString(e)), PM_EIO;
  return PM_OK;
}

inline int no_wide_kernel(const PmParams& P, const PmIO& io) {
  snprintf(pmk_g_err, sizeof pmk_g_err, "no wide kernel for nl=%d (G=%d), nterms=%d, v_mac row %d, multiplet %d, "
           "pixel grids %d", P.nl, P.G, P.K, int(P.mac_row >= 0), int(P.n_pi > 1 || P.n_sig > 1),
           int(io.lambda_pix != nullptr));
  return PM_ENOTSUP;
}

// Instances by flag for one NTERMS.  The plain combination (no multiplet, no
// v_mac row, the grid's wavelengths) is compiled only where PLAIN is set.
template <typename R, int KT, int G, int MINB, bool MAC, bool PLAIN>
int invert_wide_flags(const PmParams& P, const PmIO& io, cudaStream_t st, int num_sms, float* kernel_ms) {
  const bool zm = P.n_pi > 1 || P.n_sig > 1, pg = io.lambda_pix != nullptr;
  if constexpr (PLAIN && !MAC) {
    if (!zm && !pg) return launch_invert_wide_inst<R, KT, G, MINB, false, false, false>(P, io, st, num_sms, kernel_ms);
  } else if constexpr (!PLAIN) {
    if (zm && pg) return launch_invert_wide_inst<R, KT, G, MINB, true, MAC, true>(P, io, st, num_sms, kernel_ms);
    if (zm) return launch_invert_wide_inst<R, KT, G, MINB, true, MAC, false>(P, io, st, num_sms, kernel_ms);
    if (pg) return launch_invert_wide_inst<R, KT, G, MINB, false, MAC, true>(P, io, st, num_sms, kernel_ms);
    if constexpr (MAC) return launch_invert_wide_inst<R, KT, G, MINB, false, true, false>(P, io, st, num_sms, kernel_ms);
  }
  return no_wide_kernel(P, io);
}

// The wide inversion in one precision: FP32 at 8 (two warps per pixel) or 4
// (four) blocks per SM, FP64 at 1.  NTERMS 9 never has a v_mac row, 11 always.
template <typename R, bool PLAIN>
int invert_wide_dispatch(const PmParams& P, const PmIO& io, cudaStream_t st, int num_sms, float* kernel_ms) {
  constexpr bool f32 = sizeof(R) == 4;
  const bool mac = P.mac_row >= 0;
  if (P.G == 2) {
    if (P.K == 9) return invert_wide_flags<R, 9, 2, f32 ? 8 : 1, false, PLAIN>(P, io, st, num_sms, kernel_ms);
    if (P.K == 10 && mac) return invert_wide_flags<R, 10, 2, f32 ? 8 : 1, true, PLAIN>(P, io, st, num_sms, kernel_ms);
    if (P.K == 10) return invert_wide_flags<R, 10, 2, f32 ? 8 : 1, false, PLAIN>(P, io, st, num_sms, kernel_ms);
    if (P.K == 11) return invert_wide_flags<R, 11, 2, f32 ? 8 : 1, true, PLAIN>(P, io, st, num_sms, kernel_ms);
  } else if (P.G == 4) {
    if (P.K == 9) return invert_wide_flags<R, 9, 4, f32 ? 4 : 1, false, PLAIN>(P, io, st, num_sms, kernel_ms);
    if (P.K == 10 && mac) return invert_wide_flags<R, 10, 4, f32 ? 4 : 1, true, PLAIN>(P, io, st, num_sms, kernel_ms);
    if (P.K == 10) return invert_wide_flags<R, 10, 4, f32 ? 4 : 1, false, PLAIN>(P, io, st, num_sms, kernel_ms);
    if (P.K == 11) return invert_wide_flags<R, 11, 4, f32 ? 4 : 1, true, PLAIN>(P, io, st, num_sms, kernel_ms);
  }
  return no_wide_kernel(P, io);
}

// Synthesis instances by flag (the pixel's wavelengths are a run-time choice
// there: synthesis is not on the inversion's path).
template <typename R, int KT, int G, bool MAC, bool PLAIN>
int synth_wide_flags(const PmParams& P, const PmIO& io, cudaStream_t st) {
  const bool zm = P.n_pi > 1 || P.n_sig > 1;
  if constexpr (PLAIN && !MAC) {
    if (!zm) return launch_synth_wide_inst<R, KT, G, false, false>(P, io, st);
  } else if constexpr (!PLAIN) {
    if (zm) return launch_synth_wide_inst<R, KT, G, true, MAC>(P, io, st);
    if constexpr (MAC) return launch_synth_wide_inst<R, KT, G, false, true>(P, io, st);
  }
  return no_wide_kernel(P, io);
}

template <typename R, bool PLAIN>
int synth_wide_dispatch(const PmParams& P, const PmIO& io, cudaStream_t st) {
  const bool mac = P.mac_row >= 0;
  if (P.G == 2) {
    if (P.K == 9) return synth_wide_flags<R, 9, 2, false, PLAIN>(P, io, st);
    if (P.K == 10 && mac) return synth_wide_flags<R, 10, 2, true, PLAIN>(P, io, st);
    if (P.K == 10) return synth_wide_flags<R, 10, 2, false, PLAIN>(P, io, st);
    if (P.K == 11) return synth_wide_flags<R, 11, 2, true, PLAIN>(P, io, st);
  } else if (P.G == 4) {
    if (P.K == 9) return synth_wide_flags<R, 9, 4, false, PLAIN>(P, io, st);
    if (P.K == 10 && mac) return synth_wide_flags<R, 10, 4, true, PLAIN>(P, io, st);
    if (P.K == 10) return synth_wide_flags<R, 10, 4, false, PLAIN>(P, io, st);
    if (P.K == 11) return synth_wide_flags<R, 11, 4, true, PLAIN>(P, io, st);
  }
  return no_wide_kernel(P, io);
}

}  // namespace
