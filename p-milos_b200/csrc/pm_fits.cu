// pm_fits.cu -- cube ingest: the FITS spectro-cube header (host) and the
// reorder of its data block into the inversion layout (device).
//
// The reference reads a cube with CFITSIO and reorders it on the host
// (readFitsSpectroImage, utilsFits.c:25-368): axis roles come from CTYPE1..4
// ('HPLN-TAN' rows, 'HPLT-TAN' columns, 'WAVE-GRI' wavelength, 'STOKES'), or,
// when any CTYPE is missing, the smallest axis is Stokes, the smallest of the
// others is wavelength and the remaining two are rows then columns in axis
// order; every element lands at [pixel][stokes][lambda] with pixel =
// column * rows + row (the generic branch, utilsFits.c:242-336).  Here the raw
// big-endian data block goes to the device as it is stored in the file and one
// kernel byte-swaps and permutes it.  The reference's special branch for the
// (rows, columns, wavelength, Stokes) order (utilsFits.c:160, :228-241) indexes
// that order as if it were (wavelength, Stokes, rows, columns); this ingest
// applies the generic branch's mapping to every order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "pm_params.h"

namespace {

constexpr int kCard = 80, kBlock = 2880;

bool key_is(const char* card, const char* key) {
  const size_t n = std::strlen(key);
  if (std::strncmp(card, key, n) != 0) return false;
  for (size_t i = n; i < 8; ++i)
    if (card[i] != ' ') return false;
  return true;
}

bool card_long(const char* card, long long* v) {
  if (card[8] != '=') return false;
  char buf[72];
  std::memcpy(buf, card + 10, 70);
  buf[70] = 0;
  char* end = nullptr;
  *v = std::strtoll(buf, &end, 10);
  return end != buf;
}

// the quoted string value of a card, trailing blanks removed
bool card_string(const char* card, char* out, size_t cap) {
  if (card[8] != '=') return false;
  const char* v = card + 10;
  const char* stop = card + kCard;
  while (v < stop && *v == ' ') ++v;
  if (v >= stop || *v != '\'') return false;
  ++v;
  size_t n = 0;
  while (v < stop && n + 1 < cap) {
    if (*v == '\'') {
      if (v + 1 < stop && v[1] == '\'') {
        out[n++] = '\'';
        v += 2;
        continue;
      }
      break;
    }
    out[n++] = *v++;
  }
  while (n > 0 && out[n - 1] == ' ') --n;
  out[n] = 0;
  return true;
}

// out[((pixel * 4 + s) * nl) + l] = byteswap(in[l*st_l + s*st_s + row*st_r + col*st_c]),
// pixel = col * rows + row, i.e. out = sum over axes of coordinate * ost[axis].
// Three forms, all reading and writing coalesced, HBM-bound:
//  * identity (the reference's default order: wavelength, Stokes, rows,
//    columns): a flat byte swap, 16 bytes per thread and step;
//  * wavelength contiguous in the input: one warp per pixel, whose four Stokes
//    rows are four contiguous runs of the input and one contiguous run of the
//    output (16-byte accesses when nl is a multiple of 4); the pixel's input
//    offset advances by additions from one pixel to the next;
//  * otherwise 32 x 32 tiles of (the input's contiguous axis, wavelength), each
//    transposed by one warp through its own shared-memory tile: 32 loads in
//    flight per lane, then 32 stores, with no block barrier.
struct Reorder {
  long long n[4];    // axis sizes
  long long st[4];   // element strides of the axes in the input
  long long ost[4];  // element strides of the axes in the output
  int ax_row, ax_col, ax_l, ax_s;
  long long rows, nl, total;
};

__device__ __forceinline__ unsigned int swap32(unsigned int u) { return __byte_perm(u, 0, 0x0123); }
__device__ __forceinline__ float swap_be(unsigned int u) { return __uint_as_float(swap32(u)); }
__device__ __forceinline__ uint4 swap_be4(uint4 v) {
  v.x = swap32(v.x);
  v.y = swap32(v.y);
  v.z = swap32(v.z);
  v.w = swap32(v.w);
  return v;
}

__global__ void __launch_bounds__(256) reorder_identity(const uint4* __restrict__ in, uint4* __restrict__ out,
                                                       long long n4) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride)
    out[i] = swap_be4(__ldg(in + i));
}

// Wavelength contiguous in the input.  Each warp takes a run of `per` pixels
// (pixel = col * rows + row); within the run the pixel's input offset advances
// by st_row, and by st_col - (rows - 1) * st_row when the row wraps.  VEC: nl is
// a multiple of 4 and both arrays start on 16-byte boundaries.
template <bool VEC>
__global__ void __launch_bounds__(256) reorder_rows(const Reorder R, const unsigned int* __restrict__ in,
                                                   float* __restrict__ out, long long per) {
  const int lane = threadIdx.x & 31;
  const long long npix = R.total / (4 * R.nl);
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  const long long st_s = R.st[R.ax_s], st_row = R.st[R.ax_row], st_col = R.st[R.ax_col];
  const long long nl = R.nl;
  for (long long p0 = ((long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * per; p0 < npix;
       p0 += nwarps * per) {
    const long long p1 = p0 + per < npix ? p0 + per : npix;
    long long row = p0 % R.rows;
    long long ib = row * st_row + (p0 / R.rows) * st_col;
    for (long long p = p0; p < p1; ++p) {
      float* o = out + p * 4 * nl;
      if constexpr (VEC) {
        const long long n4 = nl >> 2;
        for (long long q = lane; q < n4; q += 32) {
          uint4 v[4];
#pragma unroll
          for (int s = 0; s < 4; ++s) v[s] = __ldg(reinterpret_cast<const uint4*>(in + ib + s * st_s) + q);
#pragma unroll
          for (int s = 0; s < 4; ++s) reinterpret_cast<uint4*>(o + s * nl)[q] = swap_be4(v[s]);
        }
      } else {
        for (long long l = lane; l < nl; l += 32) {
          unsigned int v[4];
#pragma unroll
          for (int s = 0; s < 4; ++s) v[s] = __ldg(in + ib + s * st_s + l);
#pragma unroll
          for (int s = 0; s < 4; ++s) o[s * nl + l] = swap_be(v[s]);
        }
      }
      if (++row == R.rows) {
        row = 0;
        ib += st_col - (R.rows - 1) * st_row;
      } else {
        ib += st_row;
      }
    }
  }
}

// Work item = (f segment, wavelength tile, g, h), segments consecutive: a run of
// kSegTiles 32 x 32 tiles along f, the input's contiguous axis; one warp per item
// (the item's offsets are decomposed once, not per tile; four tiles per item keep
// enough items for every warp of the grid): lane = f while loading, lane =
// wavelength while storing (the output's contiguous axis).  The 32 loads of a
// tile are unconditional, so all of them are in flight at once: a partial tile
// clamps its indices to its last row and column (those loads hit lines the tile
// reads anyway and are never stored).
constexpr int kSegTiles = 4;

__global__ void __launch_bounds__(256) reorder_tiled(const Reorder R, int f, int g, int h,
                                                    const unsigned int* __restrict__ in, float* __restrict__ out) {
  __shared__ float tile[8][32][33];
  const int x = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long nf = R.n[f], tl = (R.nl + 31) / 32;
  const long long segs = (nf + 32 * kSegTiles - 1) / (32 * kSegTiles);
  const long long items = segs * tl * R.n[g] * R.n[h];
  const long long nwarps = (long long)gridDim.x * 8;
  const long long st_l = R.st[R.ax_l], ost_f = R.ost[f];
  for (long long it = (long long)blockIdx.x * 8 + w; it < items; it += nwarps) {
    const long long sg = it % segs, r1 = it / segs;
    const long long lt = r1 % tl, r2 = r1 / tl;
    const long long cg = r2 % R.n[g], ch = r2 / R.n[g];
    const long long l0 = lt * 32;
    const int lx = int(R.nl - l0 < 32 ? R.nl - l0 : 32);
    const unsigned int* src_run = in + cg * R.st[g] + ch * R.st[h] + l0 * st_l;
    float* dst_run = out + cg * R.ost[g] + ch * R.ost[h] + l0;
    const long long f_end = (sg + 1) * 32 * kSegTiles < nf ? (sg + 1) * 32 * kSegTiles : nf;
#pragma unroll 1
    for (long long f0 = sg * 32 * kSegTiles; f0 < f_end; f0 += 32) {
      const int fx = int(nf - f0 < 32 ? nf - f0 : 32);
      const unsigned int* src = src_run + f0 + (x < fx ? x : fx - 1);
      unsigned int u[32];
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        u[k] = __ldg(src);
        if (k + 1 < lx) src += st_l;
      }
#pragma unroll
      for (int k = 0; k < 32; ++k) tile[w][k][x] = swap_be(u[k]);
      __syncwarp();
      float* dst = dst_run + f0 * ost_f + x;
#pragma unroll 8
      for (int k = 0; k < 32; ++k)
        if (k < fx && x < lx) dst[k * ost_f] = tile[w][x][k];
      __syncwarp();
    }
  }
}

}  // namespace

extern "C" int pm_fits_parse_header(const void* bytes, size_t nbytes, pm_fits_cube* out) {
  if (!bytes || !out) return pmh_fail(PM_EINVAL, "pm_fits_parse_header: NULL argument");
  std::memset(out, 0, sizeof *out);
  const char* b = static_cast<const char*>(bytes);
  long long bitpix = 0, naxis = -1, nax[4] = {0, 0, 0, 0};
  char ctype[4][72] = {{0}};
  bool have_ctype[4] = {false, false, false, false};
  bool end = false;
  size_t pos = 0;
  for (; pos + kCard <= nbytes && !end; pos += kCard) {
    const char* c = b + pos;
    if (key_is(c, "END")) {
      end = true;
      break;
    }
    long long v = 0;
    if (key_is(c, "BITPIX") && card_long(c, &v)) bitpix = v;
    else if (key_is(c, "NAXIS") && card_long(c, &v)) naxis = v;
    for (int a = 0; a < 4; ++a) {
      char k[8];
      std::snprintf(k, sizeof k, "NAXIS%d", a + 1);
      if (key_is(c, k) && card_long(c, &v)) nax[a] = v;
      std::snprintf(k, sizeof k, "CTYPE%d", a + 1);
      if (key_is(c, k)) have_ctype[a] = card_string(c, ctype[a], sizeof ctype[a]);
    }
  }
  if (!end) return pmh_fail(PM_EINVAL, "pm_fits_parse_header: no END card in the bytes given");
  if (bitpix != -32) return pmh_fail(PM_ENOTSUP, "pm_fits_parse_header: the cube must be BITPIX = -32 (float32)");
  if (naxis != 4) return pmh_fail(PM_EINVAL, "pm_fits_parse_header: the cube must have 4 axes");
  for (int a = 0; a < 4; ++a)
    if (nax[a] < 1) return pmh_fail(PM_EINVAL, "pm_fits_parse_header: bad NAXISn");
  int ax_row = -1, ax_col = -1, ax_l = -1, ax_s = -1;
  const bool header = have_ctype[0] && have_ctype[1] && have_ctype[2] && have_ctype[3];
  if (header) {
    for (int a = 0; a < 4; ++a) {
      if (!std::strcmp(ctype[a], "WAVE-GRI")) ax_l = a;
      if (!std::strcmp(ctype[a], "HPLN-TAN")) ax_row = a;
      if (!std::strcmp(ctype[a], "HPLT-TAN")) ax_col = a;
      if (!std::strcmp(ctype[a], "STOKES")) ax_s = a;
    }
    if (ax_l < 0 || ax_row < 0 || ax_col < 0 || ax_s < 0)
      return pmh_fail(PM_EINVAL, "pm_fits_parse_header: CTYPE1..4 must name WAVE-GRI, HPLN-TAN, HPLT-TAN, STOKES");
  } else {
    long long best = 10000;  // the reference's initial bound (utilsFits.c:110-127)
    for (int a = 0; a < 4; ++a)
      if (nax[a] < best) {
        ax_s = a;
        best = nax[a];
      }
    best = 10000;
    for (int a = 0; a < 4; ++a)
      if (a != ax_s && nax[a] < best) {
        ax_l = a;
        best = nax[a];
      }
    if (ax_s < 0 || ax_l < 0) return pmh_fail(PM_EINVAL, "pm_fits_parse_header: cannot infer the axis roles");
    for (int a = 0; a < 4; ++a)
      if (a != ax_s && a != ax_l) {
        if (ax_row < 0) ax_row = a;
        else ax_col = a;
      }
  }
  if (nax[ax_s] != 4) return pmh_fail(PM_EINVAL, "pm_fits_parse_header: the Stokes axis must have 4 planes");
  if (nax[ax_l] > PM_NL_MAX) return pmh_fail(PM_ERANGE, "pm_fits_parse_header: more wavelengths than PM_NL_MAX");
  out->naxis = int(naxis);
  for (int a = 0; a < 4; ++a) out->naxes[a] = nax[a];
  out->axis_row = ax_row;
  out->axis_col = ax_col;
  out->axis_lambda = ax_l;
  out->axis_stokes = ax_s;
  out->nrows = nax[ax_row];
  out->ncols = nax[ax_col];
  out->npix = nax[ax_row] * nax[ax_col];
  out->nlambda = int(nax[ax_l]);
  out->data_offset = (int64_t)((pos / kBlock + 1) * kBlock);
  out->data_bytes = 4 * nax[0] * nax[1] * nax[2] * nax[3];
  out->from_ctype = header ? 1 : 0;
  return PM_OK;
}

extern "C" int pm_fits_reorder(const pm_fits_cube* info, const void* data_dev, float* cube_dev, void* stream) {
  if (!info || !data_dev || !cube_dev) return pmh_fail(PM_EINVAL, "pm_fits_reorder: NULL argument");
  Reorder R{};
  long long st = 1;
  for (int a = 0; a < 4; ++a) {
    R.n[a] = info->naxes[a];
    R.st[a] = st;
    st *= info->naxes[a];
  }
  R.ax_row = info->axis_row;
  R.ax_col = info->axis_col;
  R.ax_l = info->axis_lambda;
  R.ax_s = info->axis_stokes;
  R.rows = info->nrows;
  R.nl = info->nlambda;
  R.total = st;
  const int roles = (1 << R.ax_row) | (1 << R.ax_col) | (1 << R.ax_l) | (1 << R.ax_s);
  if (roles != 15 || R.n[R.ax_s] != 4 || R.rows * info->ncols != info->npix || R.nl < 1 ||
      R.n[R.ax_l] != R.nl || R.n[R.ax_row] != R.rows)
    return pmh_fail(PM_EINVAL, "pm_fits_reorder: inconsistent cube description");
  R.ost[R.ax_l] = 1;
  R.ost[R.ax_s] = R.nl;
  R.ost[R.ax_row] = 4 * R.nl;
  R.ost[R.ax_col] = 4 * R.nl * R.rows;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const auto* in = static_cast<const unsigned int*>(data_dev);
  const long long cap = (long long)sms * 16;
  bool identity = true;
  for (int a = 0; a < 4; ++a) identity = identity && R.st[a] == R.ost[a];
  const bool aligned = (reinterpret_cast<uintptr_t>(data_dev) % 16 == 0) &&
                       (reinterpret_cast<uintptr_t>(cube_dev) % 16 == 0);
  if (identity && aligned) {
    const long long n4 = R.total / 4;  // the Stokes axis makes the element count a multiple of 4
    const long long blocks = std::min(cap, (n4 + 255) / 256);
    reorder_identity<<<unsigned(std::max(1LL, blocks)), 256, 0, s>>>(reinterpret_cast<const uint4*>(data_dev),
                                                                   reinterpret_cast<uint4*>(cube_dev), n4);
  } else if (R.ax_l == 0) {
    // pixels per warp: every warp of a full grid gets a few runs
    const long long npix = R.total / (4 * R.nl);
    const long long warps = cap * 8;
    const long long per = std::max(1LL, std::min(64LL, npix / (4 * warps)));
    const long long blocks = std::min(cap, (npix + 8 * per - 1) / (8 * per));
    if (R.nl % 4 == 0 && aligned)
      reorder_rows<true><<<unsigned(std::max(1LL, blocks)), 256, 0, s>>>(R, in, cube_dev, per);
    else
      reorder_rows<false><<<unsigned(std::max(1LL, blocks)), 256, 0, s>>>(R, in, cube_dev, per);
  } else {
    // f: the input's contiguous axis (axis 0); g, h: the two other non-wavelength axes
    const int f = 0;
    int g = -1, h = -1;
    for (int a = 1; a < 4; ++a)
      if (a != R.ax_l) {
        if (g < 0) g = a;
        else h = a;
      }
    // segments of kSegTiles tiles along f, one per warp
    const long long work = ((R.n[f] + 32 * kSegTiles - 1) / (32 * kSegTiles)) * ((R.nl + 31) / 32) * R.n[g] * R.n[h];
    const long long blocks = std::min(cap, (work + 7) / 8);
    reorder_tiled<<<unsigned(std::max(1LL, blocks)), 256, 0, s>>>(R, f, g, h, in, cube_dev);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char msg[160];
    std::snprintf(msg, sizeof msg, "pm_fits_reorder: %s", cudaGetErrorString(e));
    return pmh_fail(PM_EIO, msg);
  }
  return PM_OK;
}
