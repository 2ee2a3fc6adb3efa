// pm_device.cuh -- device code of the Milne-Eddington inversion kernels (sm_100a),
// shared by pm_kernels.cu, pm_wide.cu and pm_stream.cu.
//
// Mapping.  One warp inverts one pixel; lane l owns wavelength l (nl <= 32), so
// everything the reference does per wavelength in mil_sinrf / me_der runs once
// per lane with no loop.  A persistent grid pulls pixels from an atomic work
// counter, so pixels that need 3 or 50 LM iterations retire and refill
// independently.  Per-warp shared memory holds a transpose buffer for the
// response functions (lane = wavelength while they are computed, lane = profile
// while they are correlated with the PSF), the padded synthesis rows for the PSF
// correlation of the four Stokes profiles, and alpha/beta of the normal
// equations in FP64.
//
// Precision.  R = double is the plain form (every step FP64, the correctness twin
// of the reference's use_double build); R = float runs synthesis, response
// functions, PSF correlation and the normal equations in FP32.  The damped solve
// and the chi^2 acceptance test are FP64 in both.
//
// Reference map (file:line of the reference each device function restates):
//   voigt            fvoigt.c:15-80
//   synth_lane       mil_sinrf.c:46-285, funcionComponentFor_sinrf :418-449
//   psf_rows         direct_convolution(_ic) convolution.c:54-121, mil_sinrf.c:387-402
//   rf_lane          me_der.c:48-312, funcionComponentFor :536-609
//   rf_correlate     me_der.c:471-496
//   mac_*            fgauss fgauss.c:16-66, direct_convolution_double
//                    convolution.c:21-42, convCircular :125-153, mil_sinrf.c:288-357,
//                    me_der.c:314-438
//   normal_eq        covarm2 lib.c:71-116, totalParcialf/Matrixf :237-268
//   chisq            fchisqr lib.c:126-152
//   solve_*          mil_svd milosUtils.c:237-271
//   apply_delta      AplicaDelta milosUtils.c:47-115
//   check_model      check milosUtils.c:118-196
//   classical        estimacionesClasicas milosUtils.c:287-452 (+ milos.c:976-983)
//   invert_pixel     lm_mils milosUtils.c:466-635 (the pixel loop of milos.c:958-1009
//                    is the ticket loop of invert_stream_kernel, pm_stream.cu)
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stddef.h>
#include <utility>
#include <stdio.h>

#include "pm_params.h"

namespace {

constexpr int NL = 32;      // lanes: wavelengths of a one-warp pixel
constexpr int TRS = NL + 1;  // transpose row stride (odd: conflict-free column reads)
constexpr double kPi = 3.14159265358979323846264338327950288419716939937510;
constexpr double kVLight = 2.99792458e+5;
constexpr double kZeeman = 4.6686411e-13;
constexpr double kRsqrtPi = 0.5641895836;
constexpr double kGhostSigma = 1e21;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kLaneStateWords = 35;  // words of LaneState (synthesis state kept for the RFs)
constexpr int kLaneStatePad = 36;    // row stride: 16-byte rows, conflict-free 128-bit access

// Hui, Armstrong & Wray (1978) rational approximation of w(z), z = a - i v:
// numerator degree 6, monic denominator degree 7 (published coefficients).
__device__ constexpr double kP[7] = {122.607931777104326, 214.382388694706425, 181.928533092181549, 93.155580458138441,
                          30.180142196210589,  5.912626209773153,   0.564189583562615};
__device__ constexpr double kQ[7] = {122.60793177387535,  352.730625110963558, 457.334478783897737, 348.703917719495792,
                          170.354001821091472, 53.992906912940207,  10.479857114260399};

template <typename R>
__device__ __forceinline__ R taps(const PmParams& P, int j);
template <>
__device__ __forceinline__ float taps<float>(const PmParams& P, int j) { return P.taps_f[j]; }
template <>
__device__ __forceinline__ double taps<double>(const PmParams& P, int j) { return P.taps_d[j]; }
template <typename R>
__device__ __forceinline__ R omw(const PmParams& P, int k);
template <>
__device__ __forceinline__ float omw<float>(const PmParams& P, int k) { return P.omw_f[k]; }
template <>
__device__ __forceinline__ double omw<double>(const PmParams& P, int k) { return P.omw_d[k]; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// Voigt / Faraday-Voigt: H = Re w, F = Im w / 2 (fvoigt.c:15-80).  Horner in
// complex arithmetic, then a branch-free Smith (1962) division.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void voigt(R a, R v, R& h, R& f) {
  const R zr = a, zi = -v;
  R nr = R(kP[6]) * zr + R(kP[5]);
  R ni = R(kP[6]) * zi;
#pragma unroll
  for (int j = 4; j >= 0; --j) {
    const R tr = (nr * zr - ni * zi) + R(kP[j]);
    const R ti = nr * zi + ni * zr;
    nr = tr;
    ni = ti;
  }
  R dr = zr + R(kQ[6]);
  R di = zi;
#pragma unroll
  for (int j = 5; j >= 0; --j) {
    const R tr = (dr * zr - di * zi) + R(kQ[j]);
    const R ti = dr * zi + di * zr;
    dr = tr;
    di = ti;
  }
  const bool c = fabs(dr) >= fabs(di);
  const R big = c ? dr : di, small = c ? di : dr;
  const R x1 = c ? nr : ni, x2 = c ? ni : nr;
  R r, inv;
  if constexpr (sizeof(R) == 4) {
    r = __fdividef(small, big);
    inv = __frcp_rn(big + small * r);
  } else {
    r = small / big;
    inv = R(1) / (big + small * r);
  }
  const R wr = (x1 + x2 * r) * inv;
  const R wi = (c ? R(1) : R(-1)) * (x2 - x1 * r) * inv;
  h = wr;
  f = wi * R(0.5);
}

// Per-model terms shared by every wavelength (mil_sinrf.c:84-166, me_der.c:58-63).
// ZM: the line is a Zeeman multiplet (N_PI or N_SIG > 1, e.g. Fe I 6301.5,
// 5P2.0-5D2.0); otherwise a normal triplet (one component per group, e.g. Fe I
// 6173 and 6302, 5P1.0-5D0.0), whose splittings are compile-time operands.  zs is
// the shift of each group's last component, the one the response functions use
// (me_der.c:569-600 assigns rather than accumulates over components).  The FP32
// form evaluates these terms in FP32 as well.
template <typename R>
struct alignas(16) ModelTerms {
  R sin_gm, cosi, sinis, cosis, cosis_2, sina, cosa, sinda, cosda, sindi, cosdi, sinis_cosa, sinis_sina;
  R E0_2, cosi_E0_2, ulos, invLD, A, alf, oma;
  R zs[3];   // Zeeman splitting per gauss of each group, in Doppler units (nupB/nubB/nurB)
  R zsB[3];  // the same times B
  R auxCte;  // d u / d vlos (me_der.c:545)
  R invE0, sc, ss, cosi_2_E0;  // me_der.c:118-127
  R parcial, Bm;  // splitting per gauss and Lande unit in Doppler units, and B: the multiplet components
  double E0, B0, B1, ALF;
};

template <typename R, bool ZM = false>
__device__ __forceinline__ void model_terms(const PmParams& P, const double* m, ModelTerms<R>& T) {
  constexpr bool f32 = sizeof(R) == 4;
  const int lane = threadIdx.x & 31;
  T.E0 = m[0] * P.fo;
  T.B0 = m[7];
  T.B1 = -(m[8] * P.mu);
  T.ALF = m[10];
  T.alf = R(m[10]);
  T.oma = R(1.0 - m[10]);
  T.A = R(m[4]);
  // lane 0 evaluates the inclination, lane 1 the azimuth: one sincos per warp
  R s, c;
  if constexpr (f32) {
    const float CC = float(kPi / 180.0);
    const float ang = (lane & 1) ? 2.0f * (float(m[6]) * CC) : float(m[5]) * CC;
    sincosf(ang, &s, &c);
  } else {
    const double CC = kPi / 180.0;
    sincos((lane & 1) ? 2.0 * (m[6] * CC) : m[5] * CC, &s, &c);
  }
  T.sin_gm = __shfl_sync(kFull, s, 0);
  T.cosi = __shfl_sync(kFull, c, 0);
  T.sina = __shfl_sync(kFull, s, 1);
  T.cosa = __shfl_sync(kFull, c, 1);
  T.sinis = T.sin_gm * T.sin_gm;
  T.cosis = T.cosi * T.cosi;
  T.cosis_2 = (R(1) + T.cosis) / R(2);
  const R CCr = R(kPi / 180.0), CC2 = CCr * R(2);
  T.sinda = T.cosa * CC2;
  T.cosda = -T.sina * CC2;
  T.sindi = T.cosi * T.sin_gm * CC2;
  T.cosdi = -T.sin_gm * CCr;
  T.sinis_cosa = T.sinis * T.cosa;
  T.sinis_sina = T.sinis * T.sina;
  const R LD = R(m[3]), E0 = R(T.E0), l0 = R(P.lambda0);
  T.E0_2 = E0 / R(2);
  T.cosi_E0_2 = T.E0_2 * T.cosi;
  if constexpr (f32) {
    T.invLD = __frcp_rn(LD);
    T.invE0 = __frcp_rn(E0);
  } else {
    T.invLD = R(1) / LD;
    T.invE0 = R(1) / E0;
  }
  T.ulos = (R(m[2]) * l0) * T.invLD * R(1.0 / kVLight);
  const R parcial = (l0 * l0) * T.invLD * R(kZeeman);
#pragma unroll
  for (int g = 0; g < 3; ++g) {
    const int last = ZM ? (g == 0 ? P.n_pi : P.n_sig) - 1 : 0;
    T.zs[g] = parcial * R(P.nu[g][last]);
    T.zsB[g] = T.zs[g] * R(m[1]);
  }
  if constexpr (ZM) {
    T.parcial = parcial;
    T.Bm = R(m[1]);
  }
  T.auxCte = (-l0) * T.invLD * R(1.0 / kVLight);
  T.sc = E0 * T.sinis_cosa / R(2);
  T.ss = E0 * T.sinis_sina / R(2);
  T.cosi_2_E0 = E0 * T.cosi / R(2);
}

// Copy a 16-byte-aligned POD in 16-byte units (128-bit shared-memory accesses).
template <typename T>
__device__ __forceinline__ void copy16(T& dst, const T& src) {
  static_assert(sizeof(T) % 16 == 0 && alignof(T) >= 16, "copy16 needs 16-byte units");
  float4* d = reinterpret_cast<float4*>(&dst);
  const float4* s = reinterpret_cast<const float4*>(&src);
#pragma unroll
  for (int k = 0; k < int(sizeof(T) / 16); ++k) d[k] = s[k];
}

// Everything the response functions need from the synthesis at one wavelength
// (the reference keeps it in process globals between mil_sinrf and me_der).
template <typename R>
struct alignas(16) LaneState {
  R fi[3], shi[3], uu[3], H[3], F[3];
  R parcial1, parcial2, parcial3;
  R etain, etaq, etau, etav, rhoq, rhou, rhov;
  R etai, etai_2, gp1, gp2, gp3, dt, dti, g4, g5, g6;
  R pad_;
};

static_assert(sizeof(LaneState<float>) == kLaneStatePad * sizeof(float), "LaneState layout");
static_assert(sizeof(LaneState<double>) == kLaneStatePad * sizeof(double), "LaneState layout");

// ME synthesis at wavelength offset dl (mil_sinrf.c:117-285): the three Zeeman
// groups (funcionComponentFor_sinrf, mil_sinrf.c:418-449: the strength-weighted
// sum of every component's Voigt and Faraday-Voigt profiles), the propagation
// matrix, and the Unno-Rachkovsky solution.
template <typename R, bool ZM = false>
__device__ __forceinline__ void synth_lane(const PmParams& P, const ModelTerms<R>& T, double dl, LaneState<R>& s,
                                           R S[4]) {
  const R u = R(dl) * T.invLD - T.ulos;
#pragma unroll
  for (int g = 0; g < 3; ++g) {
    if constexpr (ZM) {
      const int n = g == 0 ? P.n_pi : P.n_sig;
      R fi = 0, shi = 0, uu = 0, H = 0, F = 0;
      for (int k = 0; k < n; ++k) {
        uu = u - (T.parcial * R(P.nu[g][k])) * T.Bm;
        voigt<R>(T.A, uu, H, F);
        const R we = R(P.we[g][k]);
        fi = fi + we * H;
        shi = shi + we * F * R(2);
      }
      s.fi[g] = fi;
      s.shi[g] = shi;
      s.uu[g] = uu;  // the last component's, for the response functions
      s.H[g] = H;
      s.F[g] = F;
    } else {
      const R uu = u - T.zsB[g];
      R H, F;
      voigt<R>(T.A, uu, H, F);
      const R we = R(P.we[g][0]);
      s.fi[g] = we * H;
      s.shi[g] = we * F * R(2);
      s.uu[g] = uu;
      s.H[g] = H;
      s.F[g] = F;
    }
  }
  s.parcial1 = s.fi[1] + s.fi[2];
  s.parcial2 = T.E0_2 * (s.fi[0] - s.parcial1 / R(2));
  s.parcial3 = T.E0_2 * (s.shi[0] - (s.shi[1] + s.shi[2]) / R(2));
  s.etain = T.E0_2 * (s.fi[0] * T.sinis + s.parcial1 * T.cosis_2);
  s.etaq = s.parcial2 * T.sinis_cosa;
  s.etau = s.parcial2 * T.sinis_sina;
  s.etav = (s.fi[2] - s.fi[1]) * T.cosi_E0_2;
  s.rhoq = s.parcial3 * T.sinis_cosa;
  s.rhou = s.parcial3 * T.sinis_sina;
  s.rhov = (s.shi[2] - s.shi[1]) * T.cosi_E0_2;
  s.etai = R(1) + s.etain;
  s.etai_2 = s.etai * s.etai;
  const R auxq = s.rhoq * s.rhoq, auxu = s.rhou * s.rhou, auxv = s.rhov * s.rhov;
  s.gp1 = s.etai_2 - s.etaq * s.etaq - s.etau * s.etau - s.etav * s.etav + auxq + auxu + auxv;
  s.gp3 = s.etai_2 + auxq + auxu + auxv;
  s.gp2 = s.etaq * s.rhoq + s.etau * s.rhou + s.etav * s.rhov;
  s.dt = s.etai_2 * s.gp1 - s.gp2 * s.gp2;
  s.dti = R(1) / s.dt;
  const R gp4 = s.etai_2 * s.etaq + s.etai * (s.etav * s.rhou - s.etau * s.rhov);
  const R gp5 = s.etai_2 * s.etau + s.etai * (s.etaq * s.rhov - s.etav * s.rhoq);
  const R gp6 = s.etai_2 * s.etav + s.etai * (s.etau * s.rhoq - s.etaq * s.rhou);
  s.g4 = gp4 + s.rhoq * s.gp2;
  s.g5 = gp5 + s.rhou * s.gp2;
  s.g6 = gp6 + s.rhov * s.gp2;
  const R dtiaux = R(s.dti * T.B1);
  S[0] = R(T.B0 - double(dtiaux * s.etai * s.gp3));
  S[1] = dtiaux * s.g4;
  S[2] = dtiaux * s.g5;
  S[3] = dtiaux * s.g6;
}

// Shared memory.  Per block: the PSF taps, centred and reversed, in VEC shifted
// copies so that any 32-tap window can be read with aligned 16-byte broadcast
// loads.  Per warp: the RF transpose buffer (also scratch for the synthesis
// correlation, the reduction and the eigen solver), the padded Stokes rows of
// the synthesis correlation, alpha/beta, the eigen-solver state and the model.
constexpr int XSR = 100;  // synthesis row length: 3 float4-aligned windows of 36

template <typename R>
struct alignas(16) BlockSmem {
  static constexpr int VEC = 16 / sizeof(R);
  // rv[c][u] = G[31 - (u + c) + half] (0 outside [0, nl)): for input m the
  // taps of outputs k = 0..31 are rv[c][b + k] with b + c = 31 - m, b % VEC == 0
  R rv[VEC][64 + VEC];
  // the shared stray-light profile [4][nl] (PM_SLIGHT_SHARED): lane-indexed
  // reads of the parameter block would be serialised by the constant cache
  float sl[4 * NL];
};

// State of the damped solve: the normal equations and the Jacobi rotation tables.
struct alignas(16) SolveSmem {
  double ab[PM_NTERMS_MAX * PM_NTERMS_MAX + PM_NTERMS_MAX];  // alpha (K*K) then beta (K)
  double rot[12][3];      // per index: partner, c, signed s
  int pq[6][2];           // the rotated pairs of the current round
  double delta[PM_NTERMS_MAX];
};

template <typename R>
struct alignas(16) WarpSmem {
  R tr[NL * TRS];       // response functions: [profile][lambda] (transpose buffer)
  R xs[4][XSR];         // padded Stokes rows for the synthesis PSF correlation
  SolveSmem sv;
  R ls[NL][kLaneStatePad];    // synthesis state the response functions need, per lane
  ModelTerms<R> mt;           // per-model terms of the last synthesis (uniform)
  double model[11], trial[11];
  // the streamed kernel's place in the ticket stream: kept here rather than in
  // registers while the LM loop runs
  const PmJob* job;
  unsigned long long pix;
  long long job_k;
  int grid_cur;
  int xs_dirty;  // xs holds macroturbulence data: restore its zero padding before psf_rows
  // the lock-step kernel's ticket state: the last published count seen and the
  // first ticket and pixel count of `job`
  unsigned long long avail_seen, job_t0, job_n;
  unsigned long long pad_;
};

// The 16-byte vector loads of psf_rows and rf_correlate need every per-warp
// region, every xs row and every rv row to start on a 16-byte boundary.
template <typename R>
constexpr bool smem_layout_ok() {
  return sizeof(BlockSmem<R>) % 16 == 0 && sizeof(WarpSmem<R>) % 16 == 0 &&
         offsetof(WarpSmem<R>, xs) % 16 == 0 && (XSR * sizeof(R)) % 16 == 0 &&
         offsetof(WarpSmem<R>, ls) % 16 == 0 && offsetof(WarpSmem<R>, mt) % 16 == 0 &&
         ((64 + BlockSmem<R>::VEC) * sizeof(R)) % 16 == 0;
}
static_assert(smem_layout_ok<float>(), "shared-memory layout breaks 16-byte vector loads (float)");
static_assert(smem_layout_ok<double>(), "shared-memory layout breaks 16-byte vector loads (double)");
static_assert(3 * 12 * 12 * sizeof(double) <= sizeof(float) * NL * TRS, "eigen scratch exceeds the transpose buffer");

template <typename R>
__device__ __forceinline__ void load_taps(const PmParams& P, BlockSmem<R>& bs) {
  constexpr int VEC = BlockSmem<R>::VEC;
  for (int e = threadIdx.x; e < VEC * (64 + VEC); e += blockDim.x) {
    const int c = e / (64 + VEC), u = e % (64 + VEC);
    const int j = 31 - (u + c) + P.half;
    bs.rv[c][u] = (j >= 0 && j < P.nl) ? taps<R>(P, j) : R(0);
  }
  if (P.slight_mode == PM_SLIGHT_SHARED)
    for (int e = threadIdx.x; e < 4 * NL; e += blockDim.x) bs.sl[e] = e < 4 * P.nl ? P.sl_f[e] : 0.0f;
}

// The stray-light profile a pixel mixes in: the block's copy of the shared one,
// the pixel's own row of a per-pixel cube, or none.
template <typename R>
__device__ __forceinline__ const float* slight_of(const PmParams& P, const BlockSmem<R>& bs, const float* cube,
                                                  size_t base) {
  if (P.slight_mode == PM_SLIGHT_SHARED) return bs.sl;
  if (P.slight_mode == PM_SLIGHT_PER_PIXEL && cube) return cube + base;
  return nullptr;
}

// PSF correlation of the four synthesized profiles (mil_sinrf.c:387-402,
// convolution.c:54-121): out[k] = sum_j G[j] x[k + j - nl/2], zero padding;
// Stokes I correlates Ic - I and returns Ic - result, Ic = max(I[0], I[nl-1]).
// Lane l computes outputs 4c..4c+3 (c = l & 7) of Stokes l >> 3 from one aligned
// 36-sample window: 9 vector loads and 128 FMAs whose taps are compile-time
// indexed constant operands.
template <typename R>
__device__ __forceinline__ void psf_rows(const PmParams& P, WarpSmem<R>& sm, int lane, bool valid, R S[4]) {
  const R i0 = __shfl_sync(kFull, S[0], 0), in = __shfl_sync(kFull, S[0], P.nl - 1);
  const R ic = (i0 > in) ? i0 : in;
  const int off = NL + (P.half & 3);  // data at xs[s][off + i]; off - half is a multiple of 4
#pragma unroll
  for (int s = 0; s < 4; ++s) sm.xs[s][off + lane] = valid ? (s == 0 ? ic - S[0] : S[s]) : R(0);
  __syncwarp();
  const int st = lane >> 3, c = lane & 7;
  constexpr int VEC = 16 / sizeof(R);
  const R* w0 = &sm.xs[st][off + 4 * c - P.half];
  R w[NL + 4];
#pragma unroll
  for (int t = 0; t < NL + 4; t += VEC) {
    if constexpr (VEC == 4) {
      const float4 q = *reinterpret_cast<const float4*>(w0 + t);
      w[t] = q.x; w[t + 1] = q.y; w[t + 2] = q.z; w[t + 3] = q.w;
    } else {
      const double2 q = *reinterpret_cast<const double2*>(w0 + t);
      w[t] = q.x; w[t + 1] = q.y;
    }
  }
  R acc[4] = {R(0), R(0), R(0), R(0)};
#pragma unroll
  for (int j = 0; j < NL; ++j) {
    const R g = taps<R>(P, j);
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) acc[kk] = fma(g, w[kk + j], acc[kk]);
  }
  R* o = sm.tr;  // scratch [4][NL]
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) o[st * NL + 4 * c + kk] = (st == 0) ? ic - acc[kk] : acc[kk];
  __syncwarp();
#pragma unroll
  for (int s = 0; s < 4; ++s) S[s] = valid ? o[s * NL + lane] : R(0);
  __syncwarp();
}

// ---------------------------------------------------------------------------
// Macroturbulence (the direct branch of mil_sinrf.c:288-357 and
// me_der.c:314-438).  A Gaussian of sigma = lambda0 v_mac / c over the grid,
// centred at lambda[nl/2] and normalised to unit sum (fgauss, fgauss.c:16-66),
// is correlated with the PSF when there is one (direct_convolution_double,
// convolution.c:21-42); every synthesized profile (Stokes I included, with no
// continuum padding) and every response function but S0's is then convolved
// with it circularly, and the v_mac row is the circular convolution of the
// unconvolved synthesis with the Gaussian's derivative in the form of
// me_der.c:419-421 (GMAC / v_mac ((x / sigma)^2 - 1): the normalisation is not
// differentiated).  convCircular (convolution.c:125-153) returns its result
// rotated by nl/2: out[m] = sum_t x[t] k[(m + nl/2 - t) mod nl].
//
// While a model with v_mac > 1e-4 is current, the per-warp rows xs (the padded
// input of psf_rows otherwise) hold the unconvolved synthesis [4][32] and the
// kernel and its derivative, each tripled (entry u = k[u mod nl], u < 96) so
// that the circular index m + nl/2 - t + nl is a plain offset; xs_dirty makes
// the next psf_rows restore the zero padding first.
// ---------------------------------------------------------------------------
constexpr double kMacMin = 0.0001;
constexpr int kMacSu = 0, kMacK = 4 * NL, kMacD = 7 * NL;
static_assert(kMacD + 3 * NL <= 4 * XSR, "macroturbulence data exceed the padded rows");

// Lane k's value of the kernel (and of its derivative with DERIV), through the
// PSF; dl: lane k's wavelength offset lambda_k - lambda0; scratch: 64 doubles.
template <bool DERIV>
__device__ __forceinline__ void mac_kernel(const PmParams& P, double mac, double dl, int lane, bool valid,
                                           double* scratch, double& g, double& gd) {
  const double dlc = __shfl_sync(kFull, dl, P.half);
  const double x = valid ? dl - dlc : 0.0;  // lambda_k - lambda[nl/2], exactly
  const double ild = (P.lambda0 * mac) / kVLight;
  const double a = x / ild;
  const double term = (a * a) / 2;
  g = (valid && term < 1e30) ? exp(-term) : 0.0;
  g = g / warp_sum(g);
  gd = DERIV ? g / mac * (a * a - 1.0) : 0.0;
  if (P.has_psf) {
    __syncwarp();
    scratch[lane] = g;
    if (DERIV) scratch[NL + lane] = gd;
    __syncwarp();
    double acc = 0.0, accd = 0.0;
    for (int j = 0; j < P.nl; ++j) {
      const int t = lane + j - P.half;
      if (t >= 0 && t < P.nl) {
        acc = fma(P.taps_d[j], scratch[t], acc);
        if (DERIV) accd = fma(P.taps_d[j], scratch[NL + t], accd);
      }
    }
    __syncwarp();
    g = valid ? acc : 0.0;
    gd = valid ? accd : 0.0;
  }
}

// dst[u] = k[u mod nl] for u < 96, k[l] held by lane l.
template <typename R>
__device__ __forceinline__ void mac_triple(const PmParams& P, double k, int lane, R* dst) {
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int u = lane + NL * q;
    const double v = __shfl_sync(kFull, k, u % P.nl);
    dst[u] = R(v);
  }
}

// The kernel of v_mac (and its derivative with DERIV) into xs; tr is scratch.
template <typename R, bool DERIV>
__device__ __forceinline__ void mac_prepare(const PmParams& P, WarpSmem<R>& sm, double mac, double dl, int lane,
                                            bool valid) {
  double g, gd;
  mac_kernel<DERIV>(P, mac, dl, lane, valid, reinterpret_cast<double*>(sm.tr), g, gd);
  R* xf = &sm.xs[0][0];
  mac_triple<R>(P, g, lane, xf + kMacK);
  if (DERIV) mac_triple<R>(P, gd, lane, xf + kMacD);
  if (lane == 0) sm.xs_dirty = 1;
  __syncwarp();
}

// out[s] at this lane's wavelength m: sum_t x[s][t] k[(m + nl/2 - t) mod nl] for
// the four unconvolved rows x of xs and the tripled kernel k3.
template <typename R>
__device__ __forceinline__ void mac_circular4(const PmParams& P, const R* xf, const R* k3, int lane, R out[4]) {
  R acc[4] = {R(0), R(0), R(0), R(0)};
  const R* kb = k3 + lane + P.half + P.nl;
#pragma unroll 2
  for (int t = 0; t < P.nl; ++t) {
    const R kk = kb[-t];
#pragma unroll
    for (int s = 0; s < 4; ++s) acc[s] = fma(xf[kMacSu + s * NL + t], kk, acc[s]);
  }
#pragma unroll
  for (int s = 0; s < 4; ++s) out[s] = acc[s];
}

// The 32 response-function profiles (one per lane, rows of tr) convolved
// circularly with the kernel in xs, in place.
template <typename R>
__device__ __forceinline__ void mac_rf_circular(const PmParams& P, WarpSmem<R>& sm, int lane) {
  __syncwarp();
  R* row = sm.tr + lane * TRS;
  const R* k3 = &sm.xs[0][0] + kMacK + P.half + P.nl;
  R acc[NL];
#pragma unroll
  for (int m = 0; m < NL; ++m) acc[m] = 0;
#pragma unroll 1
  for (int t = 0; t < P.nl; ++t) {
    const R xt = row[t];
    const R* kb = k3 - t;
#pragma unroll
    for (int m = 0; m < NL; ++m) acc[m] = fma(xt, kb[m], acc[m]);
  }
#pragma unroll
  for (int m = 0; m < NL; ++m) row[m] = acc[m];
  __syncwarp();
}

// Zero the padded rows again after macroturbulence data.
template <typename R>
__device__ __forceinline__ void xs_restore(WarpSmem<R>& sm, int lane) {
  for (int e = lane; e < 4 * XSR; e += 32) (&sm.xs[0][0])[e] = R(0);
  __syncwarp();
  if (lane == 0) sm.xs_dirty = 0;
  __syncwarp();
}

// Synthesis of the model at this lane's wavelength, PSF (or macroturbulence)
// and stray light included.  S gets the final (mixed) profile, Su the profile
// before the stray-light mix.  The per-model terms and this lane's synthesis
// state are left in shared memory for the response functions, as the reference
// leaves them in globals.  MAC: the kernel has a v_mac response row (NTERMS >=
// 10), so v_mac may be nonzero.  dl: this lane's wavelength offset lambda -
// lambda0 (the grid's, or the pixel's own).
template <typename R, bool MAC = false, bool ZM = false>
__device__ __forceinline__ void synthesize(const PmParams& P, WarpSmem<R>& sm, const double* m,
                                           const float* sl_pix, int lane, bool valid, double dl, R S[4], R Su[4]) {
  ModelTerms<R> T;
  LaneState<R> st;
  model_terms<R, ZM>(P, m, T);
  synth_lane<R, ZM>(P, T, dl, st, S);
  copy16(*reinterpret_cast<LaneState<R>*>(sm.ls[lane]), st);
  if (lane == 0) copy16(sm.mt, T);
  const double mac = MAC ? m[9] : 0.0;
  if (MAC && mac > kMacMin) {
    R* xf = &sm.xs[0][0];
#pragma unroll
    for (int s = 0; s < 4; ++s) xf[kMacSu + s * NL + lane] = valid ? S[s] : R(0);
    mac_prepare<R, false>(P, sm, mac, dl, lane, valid);
    R out[4];
    mac_circular4<R>(P, xf, xf + kMacK, lane, out);
#pragma unroll
    for (int s = 0; s < 4; ++s) S[s] = valid ? out[s] : R(0);
    __syncwarp();
  } else if (P.has_psf) {
    if (MAC && sm.xs_dirty) xs_restore<R>(sm, lane);
    psf_rows<R>(P, sm, lane, valid, S);
  }
#pragma unroll
  for (int s = 0; s < 4; ++s) Su[s] = S[s];
  if (P.slight_mode != PM_SLIGHT_NONE) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int idx = s * P.nl + (valid ? lane : 0);
      const R slv = R(sl_pix[idx]);  // shared profile (block copy) or the pixel's own
      S[s] = S[s] * T.alf + slv * T.oma;
    }
  }
  __syncwarp();
}

template <typename R>
__device__ __forceinline__ void load_lane_state(const WarpSmem<R>& sm, int lane, LaneState<R>& st) {
  copy16(st, *reinterpret_cast<const LaneState<R>*>(sm.ls[lane]));
}

// Response functions at this thread's wavelength (me_der.c:85-312), profile p
// stored at col[p * STRIDE]: p = r*4 + s for rows r = 0..6 (eta0, B, vlos, dopp,
// a, gamma, azimuth) and r = 7 holding RF row 8 (S1).  Row 7 of the reference
// (S0: I = 1, Q = U = V = 0) is not convolved and is added in registers later.
template <typename R, int STRIDE, bool ZM = false>
__device__ __forceinline__ void rf_lane(const PmParams& P, const ModelTerms<R>& T, const LaneState<R>& st, R* col,
                                        bool valid) {
  R dfi[3][4], dshi[3][4];
#pragma unroll
  for (int g = 0; g < 3; ++g) {
    const R we = R(P.we[g][ZM ? (g == 0 ? P.n_pi : P.n_sig) - 1 : 0]);  // the last component's
    const R uu = st.uu[g], H = st.H[g], F = st.F[g];
    const R dH_u = ((R(4) * T.A * F) - (R(2) * uu * H)) * we;
    const R dF_u = (R(kRsqrtPi) - T.A * H - R(2) * uu * F) * we;
    const R uun = -uu * T.invLD;
    dfi[g][0] = dH_u * (-T.zs[g]);
    dfi[g][1] = dH_u * T.auxCte;
    dfi[g][2] = dH_u * uun;
    dfi[g][3] = R(-2) * dF_u;
    dshi[g][0] = dF_u * (-T.zs[g]);
    dshi[g][1] = dF_u * T.auxCte;
    dshi[g][2] = dF_u * uun;
    dshi[g][3] = dH_u / R(2);
  }
  const R invE0 = T.invE0, sc = T.sc, ss = T.ss;
  const R E0_2 = T.E0_2;
  const R sindi_cosa = T.sindi * T.cosa, sindi_sina = T.sindi * T.sina;
  const R cosdi_E0_2 = E0_2 * T.cosdi;
  const R cosi_2_E0 = T.cosi_2_E0;
  const R cosis_2_E0_2 = T.cosis_2 * E0_2, sinis_E0_2 = T.sinis * E0_2;
  const R cosi_cosdi = T.cosi * T.cosdi * E0_2, sindi_E0_2 = T.sindi * E0_2;
  const R sinis_cosda = T.sinis * T.cosda, sinis_sinda = T.sinis * T.sinda;

  const R dtaux = R(T.B1) / (st.dt * st.dt);
  const R etai = st.etai, etai_2 = st.etai_2, etaq = st.etaq, etau = st.etau, etav = st.etav;
  const R rhoq = st.rhoq, rhou = st.rhou, rhov = st.rhov;
  const R etai_gp3 = etai * st.gp3;
  const R a2 = R(2) * etai;
  const R ext1 = a2 * etaq + etav * rhou - etau * rhov;
  const R ext2 = a2 * etau + etaq * rhov - etav * rhoq;
  const R ext3 = a2 * etav + etau * rhoq - etaq * rhou;
  const R ext4 = a2 * st.gp1;
#pragma unroll
  for (int il = 0; il < 7; ++il) {
    R de, dq, du, dv, rq, ru, rv;
    if (il == 0) {
      de = st.etain * invE0; dq = st.etaq * invE0; du = st.etau * invE0; dv = st.etav * invE0;
      rq = st.rhoq * invE0; ru = st.rhou * invE0; rv = st.rhov * invE0;
    } else if (il < 5) {
      const int k = il - 1;
      const R dfisum = dfi[1][k] + dfi[2][k];
      const R aux = dfi[0][k] - dfisum / R(2);
      de = dfi[0][k] * sinis_E0_2 + dfisum * cosis_2_E0_2;
      dq = aux * sc;
      du = aux * ss;
      dv = (dfi[2][k] - dfi[1][k]) * cosi_2_E0;
      const R auxr = dshi[0][k] - (dshi[1][k] + dshi[2][k]) / R(2);
      rq = auxr * sc;
      ru = auxr * ss;
      rv = (dshi[2][k] - dshi[1][k]) * cosi_2_E0;
    } else if (il == 5) {
      de = st.fi[0] * sindi_E0_2 + st.parcial1 * cosi_cosdi;
      dq = st.parcial2 * sindi_cosa;
      du = st.parcial2 * sindi_sina;
      dv = (st.fi[2] - st.fi[1]) * cosdi_E0_2;
      rq = st.parcial3 * sindi_cosa;
      ru = st.parcial3 * sindi_sina;
      rv = (st.shi[2] - st.shi[1]) * cosdi_E0_2;
    } else {
      de = 0; dv = 0; rv = 0;
      dq = st.parcial2 * sinis_cosda;
      du = st.parcial2 * sinis_sinda;
      rq = st.parcial3 * sinis_cosda;
      ru = st.parcial3 * sinis_sinda;
    }
    const R dgp1 = R(2) * (etai * de - etaq * dq - etau * du - etav * dv + rhoq * rq + rhou * ru + rhov * rv);
    const R dgp2 = rhoq * dq + etaq * rq + rhou * du + etau * ru + rhov * dv + etav * rv;
    const R d_dt = ext4 * de + etai_2 * dgp1 - R(2) * st.gp2 * dgp2;
    const R dgp3 = R(2) * (etai * de + rhoq * rq + rhou * ru + rhov * rv);
    R dI = -(((de * st.gp3 + etai * dgp3) * st.dt - d_dt * etai_gp3) * dtaux);
    const R dgp4 = de * ext1 + etai_2 * dq + etai * (rhou * dv + etav * ru - rhov * du - etau * rv);
    const R dQ = ((dgp4 + rq * st.gp2 + rhoq * dgp2) * st.dt - d_dt * st.g4) * dtaux;
    const R dgp5 = de * ext2 + etai_2 * du + etai * (rhov * dq + etaq * rv - rhoq * dv - etav * rq);
    const R dU = ((dgp5 + ru * st.gp2 + rhou * dgp2) * st.dt - d_dt * st.g5) * dtaux;
    const R dgp6 = de * ext3 + etai_2 * dv + etai * (rhoq * du + etau * rq - rhou * dq - etaq * ru);
    R dV = ((dgp6 + rv * st.gp2 + rhov * dgp2) * st.dt - d_dt * st.g6) * dtaux;
    if (il == 6) { dI = 0; dV = 0; }  // me_der.c:309-312
    col[(il * 4 + 0) * STRIDE] = valid ? dI : R(0);
    col[(il * 4 + 1) * STRIDE] = valid ? dQ : R(0);
    col[(il * 4 + 2) * STRIDE] = valid ? dU : R(0);
    col[(il * 4 + 3) * STRIDE] = valid ? dV : R(0);
  }
  // S1 (me_der.c:281-298)
  const R dti_s1 = -(st.dti * R(P.mu));
  col[(7 * 4 + 0) * STRIDE] = valid ? -dti_s1 * etai_gp3 : R(0);
  col[(7 * 4 + 1) * STRIDE] = valid ? dti_s1 * st.g4 : R(0);
  col[(7 * 4 + 2) * STRIDE] = valid ? dti_s1 * st.g5 : R(0);
  col[(7 * 4 + 3) * STRIDE] = valid ? dti_s1 * st.g6 : R(0);
}

// PSF correlation of the 32 response-function profiles, one profile per lane
// (me_der.c:471-496): out[k] = sum_m x[m] G[m - k + nl/2].  A runtime loop over
// the inputs m keeps the code small: per m one load of x[m] from the lane's own
// row and the 32 taps of all outputs as aligned broadcast vector loads.  FP32
// takes the inputs four at a time: their taps are one window of 35 consecutive
// entries of a reversed tap row (9 vector loads for 128 products instead of 32),
// which matters because all warps of a lock-step block run this loop together and
// the broadcast loads were bound by shared-memory bandwidth; every output still
// adds its products in the order of m, so the results are those of the one-input
// loop bit for bit.  Stokes-I rows correlate Ic - x with Ic = max of the row's end
// points.
template <typename R>
__device__ __forceinline__ void rf_correlate(const PmParams& P, const BlockSmem<R>& bs, WarpSmem<R>& sm,
                                             int lane) {
  constexpr int VEC = BlockSmem<R>::VEC;
  __syncwarp();
  R* row = sm.tr + lane * TRS;
  const bool isI = (lane & 3) == 0;
  const R e0 = row[0], en = row[P.nl - 1];
  const R ic = isI ? ((e0 > en) ? e0 : en) : R(0);
  if constexpr (VEC == 4) {
    // FP32: the products in pairs, one packed FMA (sm_100 f32x2) per two outputs;
    // each half of a pair rounds exactly as a scalar fma would
    float2 acc[NL / 2];
#pragma unroll
    for (int k = 0; k < NL / 2; ++k) acc[k] = make_float2(0.0f, 0.0f);
    constexpr int BLK = 4;                           // inputs per pass of the loop
    constexpr int TW = (NL + BLK - 1 + 3) & ~3;      // their taps window, whole float4s
    int m = 0;
#pragma unroll 1
    for (; m + BLK <= P.nl; m += BLK) {
      float xb[BLK];
#pragma unroll
      for (int i = 0; i < BLK; ++i) {
        const float r = row[m + i];
        xb[i] = isI ? ic - r : r;
      }
      // input m + i, output k: tap rv[c][b + k] with c + b = 31 - (m + i), i.e.
      // t[(BLK - 1 - i) + k] of the window starting at rv[c0][b0]
      const int base = 31 - m - (BLK - 1);
      const int c0 = base & (VEC - 1), b0 = base - c0;
      const float* g = bs.rv[c0] + b0;
      float t[TW];
#pragma unroll
      for (int j = 0; j < TW; j += 4) {
        const float4 q = *reinterpret_cast<const float4*>(g + j);
        t[j] = q.x;
        t[j + 1] = q.y;
        t[j + 2] = q.z;
        t[j + 3] = q.w;
      }
#pragma unroll
      for (int i = 0; i < BLK; ++i) {
        const int sh = BLK - 1 - i;
        const float2 x2 = make_float2(xb[i], xb[i]);
#pragma unroll
        for (int k = 0; k < NL; k += 2) {
          if ((sh & 1) == 0) {
            acc[k / 2] = __ffma2_rn(x2, make_float2(t[sh + k], t[sh + k + 1]), acc[k / 2]);
          } else {
            acc[k / 2].x = fmaf(xb[i], t[sh + k], acc[k / 2].x);
            acc[k / 2].y = fmaf(xb[i], t[sh + k + 1], acc[k / 2].y);
          }
        }
      }
    }
#pragma unroll 1
    for (; m < P.nl; ++m) {
      const float xm = isI ? ic - row[m] : row[m];
      const float2 x2 = make_float2(xm, xm);
      const int c = (31 - m) & (VEC - 1), b = (31 - m) - c;
      const R* g = bs.rv[c] + b;
#pragma unroll
      for (int k = 0; k < NL; k += VEC) {
        const float4 q = *reinterpret_cast<const float4*>(g + k);
        acc[k / 2] = __ffma2_rn(x2, make_float2(q.x, q.y), acc[k / 2]);
        acc[k / 2 + 1] = __ffma2_rn(x2, make_float2(q.z, q.w), acc[k / 2 + 1]);
      }
    }
#pragma unroll
    for (int k = 0; k < NL / 2; ++k) {
      row[2 * k] = isI ? ic - acc[k].x : acc[k].x;
      row[2 * k + 1] = isI ? ic - acc[k].y : acc[k].y;
    }
  } else {
    R acc[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) acc[k] = 0;
#pragma unroll 1
    for (int m = 0; m < P.nl; ++m) {
      const R xm = isI ? ic - row[m] : row[m];
      const int c = (31 - m) & (VEC - 1), b = (31 - m) - c;
      const R* g = bs.rv[c] + b;
#pragma unroll
      for (int k = 0; k < NL; k += VEC) {
        const double2 q = *reinterpret_cast<const double2*>(g + k);
        acc[k] = fma(xm, q.x, acc[k]);
        acc[k + 1] = fma(xm, q.y, acc[k + 1]);
      }
    }
#pragma unroll
    for (int k = 0; k < NL; ++k) row[k] = isI ? ic - acc[k] : acc[k];
  }
  __syncwarp();
}

// Reduce N values held by every lane across the warp; afterwards lane l holds
// the totals of entries [l*N/32, (l+1)*N/32) in v[0 .. N/32).  Recursive halving
// (31*N/32 shuffles); one template instance per stage keeps every index into v
// a compile-time constant, so v stays in registers.
template <typename T, int N, int O>
__device__ __forceinline__ void treduce_stage(T (&v)[N], int lane) {
  constexpr int half = (N * O) / 32;
  const bool up = (lane & O) != 0;
#pragma unroll
  for (int i = 0; i < half; ++i) {
    const T send = up ? v[i] : v[i + half];
    const T keep = up ? v[i + half] : v[i];
    v[i] = keep + __shfl_xor_sync(kFull, send, O);
  }
  if constexpr (O > 1) treduce_stage<T, N, O / 2>(v, lane);
}

template <typename T, int N>
__device__ __forceinline__ void transpose_reduce(T (&v)[N], int lane) {
  static_assert(N % 32 == 0, "N must be a multiple of 32");
  treduce_stage<T, N, 16>(v, lane);
}

// Response functions at this lane's wavelength after correlation, filling factor
// and FijaACeroDerivadasNoNecesarias: d[row][stokes] for rows 0..K-1.
template <typename R, int KT>
__device__ __forceinline__ void gather_rf(const PmParams& P, const WarpSmem<R>& sm, int lane, bool valid,
                                          R alf, const R Sff[4], const float* sl_pix, const R (&dmac)[4],
                                          R (&d)[KT][4]) {
  const R* col = sm.tr + lane;
#pragma unroll
  for (int r = 0; r < KT; ++r) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      R v;
      if (r < 7) v = col[(r * 4 + s) * TRS];
      else if (r == 7) v = (s == 0) ? R(1) : R(0);  // S0 (me_der.c:301-306)
      else if (r == 8) v = col[(7 * 4 + s) * TRS];
      else if (r == 9 && P.mac_row == 9) v = dmac[s];  // zero while v_mac <= 1e-4
      else v = R(0);
      d[r][s] = valid ? v : R(0);
    }
  }
  if (P.slight_mode != PM_SLIGHT_NONE) {
    // me_der.c:499-525: every RF scaled by alpha; the filling-factor row is
    // S_mag - S_stray, built from the spectrum the caller passes (Sff)
#pragma unroll
    for (int r = 0; r < KT; ++r) {
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        d[r][s] = d[r][s] * alf;
        if (r == P.ff_row) {
          const int idx = s * P.nl + (valid ? lane : 0);
          const R slv = R(sl_pix[idx]);
          d[r][s] = valid ? Sff[s] - slv : R(0);
        }
      }
    }
  }
}

// Entry e of the packed normal-equation vector: the upper triangle of alpha row
// by row (a <= b), then beta.  Constant-folded inside unrolled loops.
__host__ __device__ constexpr int ne_row(int e, int K) {
  int a = 0;
  while (a < K && e >= K - a) { e -= K - a; ++a; }
  return a;  // == K for the beta part
}
__host__ __device__ constexpr int ne_col(int e, int K) {
  int a = 0;
  while (a < K && e >= K - a) { e -= K - a; ++a; }
  return a < K ? a + e : e;
}

// One packed entry with compile-time (a, b): an alpha product or a beta term.
template <typename R, int KT, int E>
__device__ __forceinline__ R ne_entry(const R (&d)[KT][4], const R (&cw)[4], const R (&rw)[4]) {
  constexpr int NT = KT * (KT + 1) / 2 + KT;
  if constexpr (E >= NT) {
    return R(0);
  } else {
    constexpr int a = ne_row(E, KT), b = ne_col(E, KT);
    R acc = 0;
    if constexpr (a < KT) {
#pragma unroll
      for (int s = 0; s < 4; ++s) acc = fma(d[a][s] * d[b][s], cw[s], acc);
    } else {
#pragma unroll
      for (int s = 0; s < 4; ++s) acc = fma(rw[s], d[b][s], acc);
    }
    return acc;
  }
}

template <typename R, int KT, int CH, int... I>
__device__ __forceinline__ void ne_chunk(R (&v)[32], const R (&d)[KT][4], const R (&cw)[4], const R (&rw)[4],
                                         std::integer_sequence<int, I...>) {
  ((v[I] = ne_entry<R, KT, CH * 32 + I>(d, cw, rw)), ...);
}

template <typename R, int KT, int CH>
__device__ __forceinline__ void ne_reduce_chunk(double* red, int lane, const R (&d)[KT][4], const R (&cw)[4],
                                                const R (&rw)[4]) {
  R v[32];
  ne_chunk<R, KT, CH>(v, d, cw, rw, std::make_integer_sequence<int, 32>{});
  transpose_reduce<R, 32>(v, lane);
  red[CH * 32 + lane] = double(v[0]);
}

// Normal equations (covarm2): alpha = sum w_s/sigma^2 d_a d_b (upper triangle),
// beta = sum w_s (S - O)/sigma^2 d_b, reduced over the warp in chunks of 32
// entries (31 shuffles each) and stored in FP64.
template <typename R, int KT>
__device__ __forceinline__ void normal_eq(const PmParams& P, WarpSmem<R>& sm, int lane, const R (&d)[KT][4],
                                          const R S[4], const float O[4], const R isig[4]) {
  constexpr int NA = KT * (KT + 1) / 2;
  constexpr int NT = NA + KT;
  constexpr int NCH = (NT + 31) / 32;
  static_assert(NCH <= 3, "at most 96 packed entries");
  R cw[4], rw[4];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    cw[s] = R(P.w[s]) * isig[s];
    rw[s] = R(P.w[s]) * (S[s] - R(O[s])) * isig[s];
  }
  double* red = reinterpret_cast<double*>(sm.tr);  // scratch: the RFs are in registers now
  __syncwarp();
  ne_reduce_chunk<R, KT, 0>(red, lane, d, cw, rw);
  if constexpr (NCH > 1) ne_reduce_chunk<R, KT, 1>(red, lane, d, cw, rw);
  if constexpr (NCH > 2) ne_reduce_chunk<R, KT, 2>(red, lane, d, cw, rw);
  __syncwarp();
  // unpack: full symmetric alpha (K x K) and beta
  for (int e = lane; e < KT * KT + KT; e += 32) {
    double val;
    if (e < KT * KT) {
      int a = e / KT, b = e % KT;
      if (a > b) { int t = a; a = b; b = t; }
      val = red[a * KT - (a * (a - 1)) / 2 + (b - a)];
    } else {
      val = red[NA + (e - KT * KT)];
    }
    sm.sv.ab[e] = val;
  }
  __syncwarp();
}

// chi^2 / nfree (fchisqr), accumulated in FP64.
template <typename R>
__device__ __forceinline__ double chisq(const PmParams& P, const R S[4], const float O[4], const R isig[4],
                                        bool valid, double nfree) {
  double acc = 0;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const R dif = S[s] - R(O[s]);
    acc += valid ? double(dif * dif) * P.w[s] * double(isig[s]) : 0.0;
  }
  return warp_sum(acc) / nfree;
}

// ---------------------------------------------------------------------------
// Damped solve.  covar = alpha with the diagonal scaled by (1 + lambda_LM).
// ---------------------------------------------------------------------------

// Symmetric eigen-decomposition by parallel-ordered Jacobi (round-robin pairs,
// all K/2 rotations of a round applied at once), then the pseudo-inverse with
// the absolute 1e-12 eigenvalue cut of mil_svd.  Warp-cooperative; every lane
// returns delta.
template <int KT>
constexpr int eigen_scratch_doubles() {
  return 3 * ((KT + 1) & ~1) * ((KT + 1) & ~1);
}

template <int KT>
__device__ __noinline__ void solve_eigen(SolveSmem& sm, double* scratch, int lane, double flambda) {
  constexpr int M = (KT + 1) & ~1;  // padded to even; index KT (if any) is a dummy
  double* A = scratch;  // eigen_scratch_doubles<KT>() doubles, idle otherwise during the solve
  double* V = A + M * M;
  double* A2 = V + M * M;
  for (int e = lane; e < M * M; e += 32) {
    const int i = e / M, j = e % M;
    double a = 0;
    if (i < KT && j < KT) {
      a = sm.ab[i * KT + j];
      if (i == j) a *= (1.0 + flambda);
    }
    A[e] = a;
    V[e] = (i == j) ? 1.0 : 0.0;
  }
  __syncwarp();
  for (int sweep = 0; sweep < 24; ++sweep) {
    double off = 0, dg = 0;
    for (int e = lane; e < KT * KT; e += 32) {
      const int i = e / KT, j = e % KT;
      const double a = A[i * M + j];
      if (i == j) dg += a * a;
      else if (i < j) off += a * a;
    }
    off = warp_sum(off);
    dg = warp_sum(dg);
    if (off == 0.0 || off <= 1e-36 * dg) break;
    for (int r = 0; r < M - 1; ++r) {
      // circle method: position 0 fixed, positions 1..M-1 rotate
      if (lane < M / 2) {
        const int k = lane;
        const int pa = (k == 0) ? 0 : ((k - 1 + r) % (M - 1)) + 1;
        const int pb = ((M - 1 - k - 1 + r) % (M - 1)) + 1;
        const int p = pa < pb ? pa : pb, q = pa < pb ? pb : pa;
        double c = 1.0, s = 0.0, t = 0.0;
        const double apq = (p < KT && q < KT) ? A[p * M + q] : 0.0;
        if (apq != 0.0) {
          const double app = A[p * M + p], aqq = A[q * M + q];
          const double theta = (aqq - app) / (2.0 * apq);
          t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
          if (!isfinite(t)) t = 0.0;
          c = rsqrt(t * t + 1.0);
          s = t * c;
        }
        // column p of J: (c at p, -s at q); column q: (s at p, c at q)
        sm.rot[p][0] = q; sm.rot[p][1] = c; sm.rot[p][2] = -s;
        sm.rot[q][0] = p; sm.rot[q][1] = c; sm.rot[q][2] = s;
        sm.pq[k][0] = p; sm.pq[k][1] = q;
        // exact diagonal update (Rutishauser) stored in the unused slot of delta
        if (p < KT) sm.delta[p] = A[p * M + p] - t * apq;
        if (q < KT) sm.delta[q] = A[q * M + q] + t * apq;
      }
      __syncwarp();
      for (int e = lane; e < M * M; e += 32) {
        const int i = e / M, j = e % M;
        const int pi = int(sm.rot[i][0]), pj = int(sm.rot[j][0]);
        const double ci = sm.rot[i][1], si = sm.rot[i][2], cj = sm.rot[j][1], sj = sm.rot[j][2];
        double a;
        if (i == j) a = (i < KT) ? sm.delta[i] : 0.0;
        else if (pi == j) a = 0.0;
        else
          a = ci * (cj * A[i * M + j] + sj * A[i * M + pj]) + si * (cj * A[pi * M + j] + sj * A[pi * M + pj]);
        A2[e] = a;
      }
      // V <- V J, one work item per (row, rotated pair): both columns of the pair
      // are rewritten from their old values by the same lane
      for (int e = lane; e < M * (M / 2); e += 32) {
        const int i = e / (M / 2), k = e % (M / 2);
        const int p = sm.pq[k][0], q = sm.pq[k][1];
        const double vp = V[i * M + p], vq = V[i * M + q];
        V[i * M + p] = vp * sm.rot[p][1] + vq * sm.rot[p][2];
        V[i * M + q] = vq * sm.rot[q][1] + vp * sm.rot[q][2];
      }
      __syncwarp();
      for (int e = lane; e < M * M; e += 32) A[e] = A2[e];
      __syncwarp();
    }
  }
  // pseudo-inverse: aux_j = (V^T beta)_j / w_j (0 if |w_j| <= 1e-12); delta = V aux
  const double* beta = sm.ab + KT * KT;
  if (lane < KT) {
    double sum = 0;
    for (int i = 0; i < KT; ++i) sum += beta[i] * V[i * M + lane];
    const double w = A[lane * M + lane];
    sm.rot[lane][0] = sum * ((fabs(w) > 1e-12) ? (1.0 / w) : 0.0);
  }
  __syncwarp();
  if (lane < KT) {
    double sum = 0;
    for (int j = 0; j < KT; ++j) sum += V[lane * M + j] * sm.rot[j][0];
    sm.delta[lane] = sum;
  }
  __syncwarp();
}

// FP64 Cholesky solve of the damped normal equations, warp-cooperative: lane i
// owns row i.  Right-looking factorisation: the pivot and the new column of L
// travel by shuffle, one reciprocal square root per pivot (no divisions); the
// forward solve is column-oriented (lane i updates its own right-hand side);
// the back solve reads the factor from shared memory.  Every lane returns the
// step.  Exactly-zero rows (fixed parameters) get a zero step, as the
// pseudo-inverse gives them.  Returns false on a pivot <= 1e-12 (the caller
// then uses the eigen solver for this step).
template <int KT>
__device__ __forceinline__ bool solve_cholesky(SolveSmem& sm, double* scratch, int lane, double flambda,
                                               double (&delta)[KT]) {
  const int i = lane < KT ? lane : KT - 1;
  const double damp = 1.0 + flambda;
  double a[KT];
  bool zdiag = false;
#pragma unroll
  for (int k = 0; k < KT; ++k) {
    a[k] = sm.ab[i * KT + k];
    if (k == i) {
      zdiag = a[k] == 0.0;
      a[k] *= damp;
    }
  }
  const unsigned zr = __ballot_sync(kFull, lane < KT && zdiag);
  double rinv[KT];
  bool ok = true;
#pragma unroll
  for (int j = 0; j < KT; ++j) {
    const double piv = __shfl_sync(kFull, a[j], j);
    const bool skip = (zr >> j) & 1u;
    ok = ok && (skip || (piv > 1e-12 && piv < 1e300));
    const double r = skip ? 0.0 : rsqrt(piv);
    rinv[j] = r;
    const double l = a[j] * r;  // L[i][j] for i > j
#pragma unroll
    for (int k = j + 1; k < KT; ++k) {
      const double lk = __shfl_sync(kFull, l, k);  // L[k][j]
      a[k] = fma(-l, lk, a[k]);
    }
    a[j] = l;
  }
  // forward: L y = beta (lane i keeps b_i; y is uniform)
  const double* beta = sm.ab + KT * KT;
  double b = (zr >> i) & 1u ? 0.0 : beta[i];
  double y[KT];
#pragma unroll
  for (int j = 0; j < KT; ++j) {
    y[j] = __shfl_sync(kFull, b, j) * rinv[j];
    if (i > j) b = fma(-a[j], y[j], b);
  }
  // back: L^T x = y, with L^T read from shared memory (L[k][j] at lt[j*KT + k])
  double* lt = scratch;
  __syncwarp();
  if (lane < KT) {
#pragma unroll
    for (int j = 0; j < KT; ++j)
      if (j < i) lt[j * KT + i] = a[j];
  }
  __syncwarp();
#pragma unroll
  for (int j = KT - 1; j >= 0; --j) {
    double s = y[j];
#pragma unroll
    for (int k = j + 1; k < KT; ++k) s = fma(-lt[j * KT + k], delta[k], s);
    delta[j] = s * rinv[j];
  }
  __syncwarp();
  return ok;
}

// AplicaDelta (milosUtils.c:47-115): p <- p - delta for free parameters, with the
// step on B clamped to +-300 G and on gamma, azimuth to +-30 deg.
template <int KT>
__device__ __forceinline__ void apply_delta(const PmParams& P, const double* m, double (&dlt)[KT], double* out) {
  auto clamp = [](double v, double lim) { return v < -lim ? -lim : (v > lim ? lim : v); };
  if (P.fix[0]) out[0] = m[0] - dlt[0];
  if (P.fix[1]) out[1] = m[1] - clamp(dlt[1], 300.0);
  if (P.fix[2]) out[2] = m[2] - dlt[2];
  if (P.fix[3]) out[3] = m[3] - dlt[3];
  if (P.fix[4]) out[4] = m[4] - dlt[4];
  if (P.fix[5]) out[5] = m[5] - clamp(dlt[5], 30.0);
  if (P.fix[6]) out[6] = m[6] - clamp(dlt[6], 30.0);
  if (P.fix[7]) out[7] = m[7] - dlt[7];
  if (P.fix[8]) out[8] = m[8] - dlt[8];
  if constexpr (KT == 11) {
    if (P.fix[9]) out[9] = m[9] - dlt[9];
    if (P.fix[10]) out[10] = m[10] - dlt[10];
  } else if constexpr (KT == 10) {
    if (P.fix[9]) out[9] = m[9] - dlt[9];     // NTERMS == 10 with v_mac inverted (then fix[10] == 0)
    if (P.fix[10]) out[10] = m[10] - dlt[9];  // NTERMS == 10 with alpha inverted (then fix[9] == 0)
  }
}

// check (milosUtils.c:118-196).
__device__ __forceinline__ void check_model(double* m) {
  if (m[1] < 0) { m[1] = -m[1]; m[5] = 180.0 - m[5]; }
  if (m[1] > 5000) m[1] = 5000;
  if (m[5] < 0) m[5] = -m[5];
  if (m[5] > 180) m[5] = 360.0 - m[5];
  if (m[6] < 0) m[6] = 180 + m[6];
  if (m[6] > 180) m[6] = m[6] - 180.0;
  if (m[0] < 1) m[0] = 1;
  if (m[0] > 2500) m[0] = 2500;
  if (m[2] < -20) m[2] = -20;
  if (m[2] > 20) m[2] = 20;
  if (m[3] < 0.0001) m[3] = 0.0001;
  if (m[3] > 0.6) m[3] = 0.6;
  if (m[4] < 0.0001) m[4] = 0.0001;
  if (m[4] > 10.0) m[4] = 10.0;
  if (m[7] < 0.0001) m[7] = 0.0001;
  if (m[7] > 2.00) m[7] = 2.00;
  if (m[8] < 0.0001) m[8] = 0.0001;
  if (m[8] > 2.00) m[8] = 2.00;
  if (m[9] < 0) m[9] = 0;
  if (m[9] > 4) m[9] = 4;
  if (m[10] < 0) m[10] = 0.0;
  if (m[10] > 1.0) m[10] = 1.0;
}

// estimacionesClasicas (milosUtils.c:287-452, forInitialUse = 1) followed by the
// NaN fixes of the drivers (milos.c:976-983) -- or, in the classical-estimates-
// only mode (P.miter < 0, milos.c:486-501), forInitialUse = 0 and no NaN fixes --
// in two halves around the sums over
// wavelengths (accumulated in FP64): the terms at one wavelength w, between the
// leading and trailing ghost wavelengths [begin, end), with Ic = I[end - 1] ...
__device__ __forceinline__ void classical_terms(const PmParams& P, const float O[4], int w, double dlw, bool valid,
                                                int begin, int end, double Ic, double (&v)[10]) {
  const double dl = valid ? dlw : 0.0;  // lambda_w - lambda0
  const bool in = valid && w >= begin && w < end - 1;
  const bool iv = in && O[0] > -1.0f && O[3] > -1.0f;
  const double a = iv ? Ic - double(O[0] + O[3]) : 0.0;
  const double av = iv ? Ic - double(O[0]) : 0.0;
  const double am = iv ? Ic - double(O[0] - O[3]) : 0.0;
  v[0] = a * dl;
  v[1] = a;
  v[2] = av * dl;
  v[3] = av;
  v[4] = am * dl;
  v[5] = am;
  const bool iq = in && O[1] > -1.0f && O[2] > -1.0f && O[3] > -1.0f;
  double gx = 0, gy = 0;
  if (iq) {
    const double L = fabs(sqrt(double(O[1]) * O[1] + double(O[2]) * O[2]));
    const double mm = fabs(4 * dl * L);
    gx = fabs(double(O[3])) * mm;
    gy = fabs(double(O[3])) * fabs(double(O[3]));
  }
  v[6] = gx;
  v[7] = gy;
  const bool iu = valid && O[2] > -1.0f && O[1] > -1.0f && (fabs(O[2]) > 0.0001f || fabs(O[1]) > 0.0001f);
  v[8] = iu ? double(O[2]) : 0.0;
  v[9] = iu ? double(O[1]) : 0.0;
}

// ... and the estimates from the ten sums.  CE: compiled with the classical-
// estimates-only branch (the pre-pass kernels; the LM kernels never run it).
template <bool CE = false>
__device__ __forceinline__ void classical_finish(const PmParams& P, const double (&v)[10], double* m) {
  const bool ce = CE && P.miter < 0;
  const double x = v[0], y = v[1], xv = v[2], yv = v[3], xm = v[4], ym = v[5];
  const double lp = fabs(y) > 1e-15 ? x / y : 0.0;
  const double lmn = fabs(ym) > 1e-15 ? xm / ym : 0.0;
  const double C = kZeeman * (P.lambda0 * P.lambda0) * P.geff;
  const double Blos = (1 / C) * ((lp - lmn) / 2);
  double Vlos = (kVLight / P.lambda0) * ((xv / yv) / 2);
  const double sx = v[6];
  const double sy = v[7] * fabs(3 * C * Blos);
  const double tan_gamma = fabs(sqrt(sx / sy));
  double gamma_rad = atan(tan_gamma);
  double gamma = gamma_rad * (180 / kPi);
  if (!ce) {  // forInitialUse (milosUtils.c:395-402)
    if (gamma >= 85 && gamma <= 90) gamma_rad = 85 * (kPi / 180);
    if (gamma > 90 && gamma <= 95) gamma_rad = 95 * (kPi / 180);
  }
  if (Blos < 0) gamma = 180 - gamma;
  const double su = v[8], sq = v[9];
  double phi = (atan(su / sq) * 180 / kPi) / 2;
  if (su > 0 && sq > 0) phi = phi;
  else if (su < 0 && sq > 0) phi = phi + 180;
  else if (su < 0 && sq < 0) phi = phi + 90;
  else if (su > 0 && sq < 0) phi = phi + 90;
  const double B_aux = fabs(Blos / cos(gamma_rad));
  if (Vlos < -4) Vlos = -4;
  if (Vlos > 4) Vlos = 4;
  m[1] = B_aux > 4000 ? 4000 : B_aux;
  m[2] = Vlos;
  m[5] = gamma;
  m[6] = phi;
  if (ce) {
    m[7] = Blos;  // milosUtils.c:449-450
    return;
  }
  if (isnan(m[1])) m[1] = 1;
  if (isnan(m[2])) m[2] = 1e-3;
  if (isnan(m[5])) m[5] = 1;
  if (isnan(m[6])) m[6] = 1;
}

// Classical estimates of a one-warp pixel (lane = wavelength, dl its offset).
template <bool CE = false>
__device__ __forceinline__ void classical(const PmParams& P, const float O[4], int lane, bool valid, double dl,
                                          double* m) {
  const int nl = P.nl;
  const unsigned neg = __ballot_sync(kFull, valid && O[0] < 0.0f);
  const unsigned validm = (nl >= 32) ? kFull : ((1u << nl) - 1u);
  // leading and trailing ghost wavelengths (I < 0)
  const unsigned nonneg = validm & ~neg;
  if (nonneg == 0) return;  // every intensity negative: no estimate possible
  const int begin = __ffs(nonneg) - 1;
  const int end = 32 - __clz(nonneg);  // one past the last non-negative
  const double Ic = __shfl_sync(kFull, double(O[0]), end - 1);
  double v[10];
  classical_terms(P, O, lane, dl, valid, begin, end, Ic, v);
#pragma unroll
  for (int i = 0; i < 10; ++i) v[i] = warp_sum(v[i]);
  classical_finish<CE>(P, v, m);
}

// The response functions of model m at this lane's wavelength (rows 0..K-1,
// before FijaACeroDerivadasNoNecesarias): me_der's rows, their PSF or
// macroturbulence convolutions, the v_mac row and the filling-factor terms.
// m must be the model of the last synthesis.  MAC: compiled with the
// macroturbulence branch (the grid has a v_mac row; NTERMS >= 10).
template <typename R, int KT, bool MAC = (KT >= 10), bool ZM = false>
__device__ __forceinline__ void response_rows(const PmParams& P, const BlockSmem<R>& bs, WarpSmem<R>& sm, int lane,
                                              bool valid, const double* m, double dl, const R Sff[4],
                                              const float* sl_pix, R (&d)[KT][4]) {
  const bool mac_on = MAC && m[9] > kMacMin;
  if (mac_on) mac_prepare<R, true>(P, sm, m[9], dl, lane, valid);  // before tr fills up
  R alf;
  {
    ModelTerms<R> T;
    copy16(T, sm.mt);
    LaneState<R> st;
    load_lane_state<R>(sm, lane, st);
    rf_lane<R, TRS, ZM>(P, T, st, sm.tr + lane, valid);
    alf = T.alf;
  }
  R dmac[4] = {R(0), R(0), R(0), R(0)};
  if (mac_on) {
    mac_rf_circular<R>(P, sm, lane);
    const R* xf = &sm.xs[0][0];
    mac_circular4<R>(P, xf, xf + kMacD, lane, dmac);
  } else if (P.has_psf) {
    rf_correlate<R>(P, bs, sm, lane);
  }
  __syncwarp();
  gather_rf<R, KT>(P, sm, lane, valid, alf, Sff, sl_pix, dmac, d);
}

// Response functions at the current synthesis -> alpha, beta in shared memory.
template <typename R, int KT, bool MAC, bool ZM>
__device__ __forceinline__ void rf_and_normal_eq(const PmParams& P, const BlockSmem<R>& bs, WarpSmem<R>& sm,
                                                 int lane, bool valid, double dl, const R S[4], const R Sff[4],
                                                 const float O[4], const R isig[4], const float* sl_pix) {
  R d[KT][4];
  response_rows<R, KT, MAC, ZM>(P, bs, sm, lane, valid, sm.model, dl, Sff, sl_pix, d);
#pragma unroll
  for (int r = 0; r < KT; ++r)
    if (P.zero_row[r]) {
#pragma unroll
      for (int s = 0; s < 4; ++s) d[r][s] = 0;
    }
  normal_eq<R, KT>(P, sm, lane, d, S, O, isig);
}

template <typename R>
__device__ __forceinline__ WarpSmem<R>& warp_smem(unsigned char* raw, int warp) {
  return reinterpret_cast<WarpSmem<R>*>(raw + sizeof(BlockSmem<R>))[warp];
}

// A pointer field of a job descriptor, read from L2 (the host may have written
// the descriptor while the kernel runs).
template <typename T>
__device__ __forceinline__ T* ld_ptr(T* const* p) {
  return reinterpret_cast<T*>(__ldcg(reinterpret_cast<const unsigned long long*>(p)));
}

// lm_mils for one pixel on one warp (milosUtils.c:466-635), starting from the
// classical estimates (milos.c:958-983): those of the pre-pass kernel when the
// whole cube was on the device before the launch, else computed here.  The
// profiles may have been written by a copy engine while the kernel runs, so
// they are read from L2.
// Pixel sm.pix of job *sm.job.  The job, the pixel index and the buffer
// pointers are read from shared memory and the descriptor where they are used,
// so that none of them occupies registers across the LM loop.
// MAC: compiled with the macroturbulence branch (grids with a v_mac row).
// PIXGRID: the pixel has its own wavelengths (the job's lambda, [npix][nl]),
// kept in a register; otherwise the grid's offsets are read from the
// parameter block where they are used.
// ZM: the line is a Zeeman multiplet.
template <typename R, int KT, bool MAC, bool PIXGRID, bool ZM = false>
__device__ __forceinline__ void invert_pixel(const PmParams& P, const BlockSmem<R>& bs, WarpSmem<R>& sm, int lane,
                                             unsigned long long* ctr) {
  const bool valid = lane < P.nl;
  double* m = sm.model;
  double* trial = sm.trial;
  const PmJob* jp = sm.job;
  size_t p = sm.pix;
  size_t base = p * 4 * P.nl;
  const float* sl_pix =
      slight_of<R>(P, bs, P.slight_mode == PM_SLIGHT_PER_PIXEL ? ld_ptr(&jp->slight) : nullptr, base);
  const float* obs = ld_ptr(&jp->spectro) + base;
  const double* model_in = ld_ptr(&jp->model_in);
  double dlp = 0.0;
  if constexpr (PIXGRID) dlp = valid ? __ldcg(ld_ptr(&jp->lambda) + p * P.nl + lane) - P.lambda0 : 0.0;
  auto dl = [&]() -> double {
    if constexpr (PIXGRID) return dlp;
    else return P.dl[valid ? lane : 0];
  };

  float O[4];
  R isig[4];
  int ghosts = 0;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    O[s] = valid ? __ldcg(obs + s * P.nl + lane) : 0.0f;
    const bool g = valid && O[s] <= -1.0f;
    ghosts += __popc(__ballot_sync(kFull, g));
    isig[s] = R(1.0 / (g ? kGhostSigma : P.noise));
  }
  if (model_in) {
    if (lane < 11) m[lane] = __ldcg(model_in + p * 11 + lane);
  } else {
    double g[11];
#pragma unroll
    for (int i = 0; i < 11; ++i) g[i] = P.guess[i];
    if (P.classical) classical(P, O, lane, valid, dl(), g);
    double mine = g[0];
#pragma unroll
    for (int i = 1; i < 11; ++i)
      if (lane == i) mine = g[i];
    if (lane < 11) m[lane] = mine;
  }
  __syncwarp();

  const int nfree = P.nfree_base - ghosts;
  int status = PM_PIX_MAXITER, iter = 0, accepted = 0, fallbacks = 0;
  double ochi = 0;
  R S[4];
  if (nfree == 0) {
    status = PM_PIX_NFREE;
    iter = -1;
#pragma unroll
    for (int s = 0; s < 4; ++s) S[s] = 0;
  } else {
    // The first pass synthesizes the starting model (trial = model) and takes
    // it as accepted without a step: one copy of the synthesis and of the
    // response functions in the loop body instead of two (instruction fetch
    // bounds this kernel), with lm_mils' order of operations unchanged.
    double chi0 = 0, flambda = P.ilambda, factor = 1.0;
    if (lane < 11) trial[lane] = m[lane];
    __syncwarp();
    bool stop = false, first = true;
    while (true) {
      if (!first) {
        double dlt[KT];
        bool ok = true;
        double* scratch = reinterpret_cast<double*>(sm.tr);  // the transpose buffer is idle here
        if (P.solver == PM_SOLVE_CHOLESKY) ok = solve_cholesky<KT>(sm.sv, scratch, lane, flambda, dlt);
        if (P.solver != PM_SOLVE_CHOLESKY || !ok) {
          if (P.solver == PM_SOLVE_CHOLESKY) ++fallbacks;
          solve_eigen<KT>(sm.sv, scratch, lane, flambda);  // step in sm.sv.delta
#pragma unroll
          for (int i = 0; i < KT; ++i) dlt[i] = sm.sv.delta[i];
          __syncwarp();
        }
        // every lane forms the (uniform) trial model; lane i stores parameter i
        double t[11];
#pragma unroll
        for (int i = 0; i < 11; ++i) t[i] = trial[i];
        apply_delta<KT>(P, m, dlt, t);
        check_model(t);
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 11; ++i)
          if (lane == i) trial[i] = t[i];
        __syncwarp();
      }
      R Su[4];
      synthesize<R, MAC, ZM>(P, sm, trial, sl_pix, lane, valid, dl(), S, Su);
      const double chi = chisq<R>(P, S, O, isig, valid, double(nfree));
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
        if (lane < 11) m[lane] = trial[lane];
        __syncwarp();
        // the filling-factor row is built from the unmixed synthesis on the
        // first call of me_der and from the mixed one after a step
        // (milosUtils.c:537 vs :587)
        R Sff[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) Sff[s] = first ? Su[s] : S[s];
        rf_and_normal_eq<R, KT, MAC, ZM>(P, bs, sm, lane, valid, dl(), S, Sff, O, isig, sl_pix);
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
    bool finite = isfinite(ochi);
#pragma unroll
    for (int i = 0; i < 11; ++i) finite = finite && isfinite(m[i]);
    if (!finite) status = PM_PIX_NONFINITE;
  }
  // outputs
  jp = *reinterpret_cast<const PmJob* const volatile*>(&sm.job);
  p = *reinterpret_cast<const volatile unsigned long long*>(&sm.pix);
  base = p * 4 * P.nl;
  if (lane < 11) ld_ptr(&jp->models)[p * 11 + lane] = m[lane];
  if (lane == 0) {
    ld_ptr(&jp->chisq)[p] = float(ochi);
    ld_ptr(&jp->iters)[p] = iter;
    int* st = ld_ptr(&jp->status);
    if (st) st[p] = status;
    atomicAdd(&ctr[PMC_ITERS], (unsigned long long)(iter > 0 ? iter : 0));
    atomicAdd(&ctr[PMC_ACCEPTED], (unsigned long long)accepted);
    if (fallbacks) atomicAdd(&ctr[PMC_FALLBACK], (unsigned long long)fallbacks);
  }
  float* spectra = ld_ptr(&jp->spectra);
  if (spectra && valid) {
#pragma unroll
    for (int s = 0; s < 4; ++s) spectra[base + s * P.nl + lane] = float(S[s]);
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// lm_mils in phases, for kernels whose warps advance in lock-step: the state of
// one pixel's LM loop lives in registers (PixelLM) between three phases that a
// block runs together, separated by block barriers -- the damped solve, the
// synthesis with chi^2 and the acceptance test, the response functions with the
// normal equations (accepted steps) -- so that at any time every warp of the
// block executes the same phase's code.  Per pixel the arithmetic and its order
// are those of invert_pixel.
// ---------------------------------------------------------------------------
template <typename R>
struct PixelLM {
  float O[4];
  R isig[4];
  R S[4], Su[4];
  const float* sl_pix;
  double dlp;
  double ochi, chi0, chi, flambda, factor;
  int nfree, status, iter, accepted, fallbacks;
  bool stop, first, accept, finished;
};

// Before the loop (invert_pixel up to its first pass): the pixel's profiles,
// ghosts, starting model; finished at once when nfree == 0.
template <typename R, bool PIXGRID>
__device__ __forceinline__ void lm_begin(const PmParams& P, const BlockSmem<R>& bs, WarpSmem<R>& sm, int lane,
                                         PixelLM<R>& L) {
  const bool valid = lane < P.nl;
  double* m = sm.model;
  const PmJob* jp = sm.job;
  const size_t p = sm.pix;
  const size_t base = p * 4 * P.nl;
  L.sl_pix = slight_of<R>(P, bs, P.slight_mode == PM_SLIGHT_PER_PIXEL ? ld_ptr(&jp->slight) : nullptr, base);
  const float* obs = ld_ptr(&jp->spectro) + base;
  const double* model_in = ld_ptr(&jp->model_in);
  L.dlp = 0.0;
  if constexpr (PIXGRID) L.dlp = valid ? __ldcg(ld_ptr(&jp->lambda) + p * P.nl + lane) - P.lambda0 : 0.0;
  const double dl = PIXGRID ? L.dlp : P.dl[valid ? lane : 0];
  int ghosts = 0;
  if ((reinterpret_cast<uintptr_t>(obs) & 15) == 0) {
    // the pixel's 4 x nl floats as nl 16-byte loads (one per lane, one
    // instruction for the warp), redistributed to lane = wavelength through the
    // warp's transpose buffer (idle while a pixel starts)
    float* stage = reinterpret_cast<float*>(sm.tr);
    if (lane < P.nl) reinterpret_cast<float4*>(stage)[lane] = __ldcg(reinterpret_cast<const float4*>(obs) + lane);
    __syncwarp();
#pragma unroll
    for (int s = 0; s < 4; ++s) L.O[s] = valid ? stage[s * P.nl + lane] : 0.0f;
    __syncwarp();
  } else {
#pragma unroll
    for (int s = 0; s < 4; ++s) L.O[s] = valid ? __ldcg(obs + s * P.nl + lane) : 0.0f;
  }
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const bool g = valid && L.O[s] <= -1.0f;
    ghosts += __popc(__ballot_sync(kFull, g));
    L.isig[s] = R(1.0 / (g ? kGhostSigma : P.noise));
  }
  if (model_in) {
    if (lane < 11) m[lane] = __ldcg(model_in + p * 11 + lane);
  } else {
    double g[11];
#pragma unroll
    for (int i = 0; i < 11; ++i) g[i] = P.guess[i];
    if (P.classical) classical(P, L.O, lane, valid, dl, g);
    double mine = g[0];
#pragma unroll
    for (int i = 1; i < 11; ++i)
      if (lane == i) mine = g[i];
    if (lane < 11) m[lane] = mine;
  }
  __syncwarp();
  L.nfree = P.nfree_base - ghosts;
  L.status = PM_PIX_MAXITER;
  L.iter = 0;
  L.accepted = 0;
  L.fallbacks = 0;
  L.ochi = 0;
  L.chi0 = 0;
  L.chi = 0;
  L.flambda = P.ilambda;
  L.factor = 1.0;
  L.stop = false;
  L.first = true;
  L.accept = false;
  L.finished = false;
  if (L.nfree == 0) {
    L.status = PM_PIX_NFREE;
    L.iter = -1;
#pragma unroll
    for (int s = 0; s < 4; ++s) L.S[s] = 0;
    L.finished = true;
  } else {
    if (lane < 11) sm.trial[lane] = m[lane];
    __syncwarp();
  }
}

// Phase 1: the damped solve and the trial model (every pass but the first).
template <typename R, int KT>
__device__ __forceinline__ void lm_solve(const PmParams& P, WarpSmem<R>& sm, int lane, PixelLM<R>& L) {
  if (L.first) return;
  double dlt[KT];
  bool ok = true;
  double* scratch = reinterpret_cast<double*>(sm.tr);
  if (P.solver == PM_SOLVE_CHOLESKY) ok = solve_cholesky<KT>(sm.sv, scratch, lane, L.flambda, dlt);
  if (P.solver != PM_SOLVE_CHOLESKY || !ok) {
    if (P.solver == PM_SOLVE_CHOLESKY) ++L.fallbacks;
    solve_eigen<KT>(sm.sv, scratch, lane, L.flambda);
#pragma unroll
    for (int i = 0; i < KT; ++i) dlt[i] = sm.sv.delta[i];
    __syncwarp();
  }
  double t[11];
#pragma unroll
  for (int i = 0; i < 11; ++i) t[i] = sm.trial[i];
  apply_delta<KT>(P, sm.model, dlt, t);
  check_model(t);
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 11; ++i)
    if (lane == i) sm.trial[i] = t[i];
  __syncwarp();
}

// Phase 2: synthesis of the trial model, chi^2, the stopping and acceptance tests.
template <typename R, bool MAC, bool PIXGRID, bool ZM>
__device__ __forceinline__ void lm_synth(const PmParams& P, WarpSmem<R>& sm, int lane, PixelLM<R>& L) {
  const bool valid = lane < P.nl;
  const double dl = PIXGRID ? L.dlp : P.dl[valid ? lane : 0];
  synthesize<R, MAC, ZM>(P, sm, sm.trial, L.sl_pix, lane, valid, dl, L.S, L.Su);
  L.chi = chisq<R>(P, L.S, L.O, L.isig, valid, double(L.nfree));
  L.accept = true;
  if (!L.first) {
    if ((fabs((L.ochi - L.chi) * 100 / L.chi) < P.toplim) || (L.chi < 0.0001)) {
      L.stop = true;
      L.status = PM_PIX_CONVERGED;
    }
    L.accept = L.chi - L.ochi < 0.;
  }
}

// Phase 3: on acceptance the response functions and normal equations at the
// new model; the damping update and the loop's end test.
template <typename R, int KT, bool MAC, bool PIXGRID, bool ZM>
__device__ __forceinline__ void lm_update(const PmParams& P, const BlockSmem<R>& bs, WarpSmem<R>& sm, int lane,
                                          PixelLM<R>& L) {
  const bool valid = lane < P.nl;
  const double dl = PIXGRID ? L.dlp : P.dl[valid ? lane : 0];
  if (L.accept) {
    if (!L.first) L.flambda = L.flambda / (5.0 * L.factor);
    if (lane < 11) sm.model[lane] = sm.trial[lane];
    __syncwarp();
    R Sff[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) Sff[s] = L.first ? L.Su[s] : L.S[s];
    rf_and_normal_eq<R, KT, MAC, ZM>(P, bs, sm, lane, valid, dl, L.S, Sff, L.O, L.isig, L.sl_pix);
    L.ochi = L.chi;
    if (L.first) L.chi0 = L.chi;
    else ++L.accepted;
  } else {
    L.flambda = L.flambda * 10.0 * L.factor;
  }
  if (!L.first) {
    if ((L.flambda > 1e+7) || (L.flambda < 1e-25)) {
      if (!L.stop) L.status = PM_PIX_LAMBDA;
      L.stop = true;
    }
    ++L.iter;
    if (P.logclambda) L.factor = double(log10f(float(L.chi)) / log10f(float(L.chi0)));
    if (!(L.iter < P.miter && !L.stop)) L.finished = true;
  }
  L.first = false;
}

// After the loop: the finite check and the pixel's results (invert_pixel's outputs).
template <typename R>
__device__ __forceinline__ void lm_end(const PmParams& P, WarpSmem<R>& sm, int lane, PixelLM<R>& L,
                                       unsigned long long* ctr) {
  const bool valid = lane < P.nl;
  double* m = sm.model;
  if (L.nfree != 0) {
    bool finite = isfinite(L.ochi);
#pragma unroll
    for (int i = 0; i < 11; ++i) finite = finite && isfinite(m[i]);
    if (!finite) L.status = PM_PIX_NONFINITE;
  }
  const PmJob* jp = *reinterpret_cast<const PmJob* const volatile*>(&sm.job);
  const size_t p = *reinterpret_cast<const volatile unsigned long long*>(&sm.pix);
  const size_t base = p * 4 * P.nl;
  if (lane < 11) ld_ptr(&jp->models)[p * 11 + lane] = m[lane];
  if (lane == 0) {
    ld_ptr(&jp->chisq)[p] = float(L.ochi);
    ld_ptr(&jp->iters)[p] = L.iter;
    int* st = ld_ptr(&jp->status);
    if (st) st[p] = L.status;
    atomicAdd(&ctr[PMC_ITERS], (unsigned long long)(L.iter > 0 ? L.iter : 0));
    atomicAdd(&ctr[PMC_ACCEPTED], (unsigned long long)L.accepted);
    if (L.fallbacks) atomicAdd(&ctr[PMC_FALLBACK], (unsigned long long)L.fallbacks);
  }
  float* spectra = ld_ptr(&jp->spectra);
  if (spectra && valid) {
#pragma unroll
    for (int s = 0; s < 4; ++s) spectra[base + s * P.nl + lane] = float(L.S[s]);
  }
  __syncwarp();
}

}  // namespace

// Text of the last launch error (defined in pm_kernels.cu).
extern char pmk_g_err[256];
