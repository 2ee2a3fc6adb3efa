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
// pixel = col * rows + row.  Wavelength is the fastest axis of the output; when
// it is also the fastest of the input (the reference's default order) every
// thread copies one element with coalesced reads and writes; otherwise a 32 x
// 32 tile of (wavelength, the input's fastest axis) goes through shared memory
// so that both sides stay coalesced.
struct Reorder {
  long long n[4];    // axis sizes
  long long st[4];   // element strides of the axes in the input
  int ax_row, ax_col, ax_l, ax_s;
  long long rows, nl, total;
};

__device__ __forceinline__ float swap_be(unsigned int u) { return __uint_as_float(__byte_perm(u, 0, 0x0123)); }

__global__ void __launch_bounds__(256) reorder_direct(const Reorder R, const unsigned int* __restrict__ in,
                                                     float* __restrict__ out) {
  // wavelength is axis 0 of the input: walk the output linearly
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < R.total; o += stride) {
    const long long l = o % R.nl;
    const long long ps = o / R.nl;
    const long long s = ps & 3, pixel = ps >> 2;
    const long long row = pixel % R.rows, col = pixel / R.rows;
    const long long i = l + s * R.st[R.ax_s] + row * R.st[R.ax_row] + col * R.st[R.ax_col];
    out[o] = swap_be(__ldg(in + i));
  }
}

// Tiled form: axis f (stride 1 in the input, not wavelength) x wavelength.
// blockIdx.x: tiles of (f, wavelength); blockIdx.y: the two remaining axes.
__global__ void __launch_bounds__(256) reorder_tiled(const Reorder R, int f, int g, int h,
                                                    const unsigned int* __restrict__ in, float* __restrict__ out) {
  __shared__ float tile[32][33];
  const long long tf = (R.n[f] + 31) / 32;
  const long long tl = (R.nl + 31) / 32;
  const long long ntile = tf * tl;
  const long long gh = R.n[g] * R.n[h];
  for (long long t = blockIdx.x; t < ntile * gh; t += gridDim.x) {
    const long long tile_id = t % ntile, rest = t / ntile;
    const long long f0 = (tile_id % tf) * 32, l0 = (tile_id / tf) * 32;
    const long long cg = rest % R.n[g], chh = rest / R.n[g];
    const long long base = cg * R.st[g] + chh * R.st[h];
    // load: threads along f (the input's contiguous axis)
    for (int k = threadIdx.x >> 5; k < 32; k += blockDim.x >> 5) {
      const long long fi = f0 + (threadIdx.x & 31), li = l0 + k;
      float v = 0.f;
      if (fi < R.n[f] && li < R.nl) v = swap_be(__ldg(in + base + fi + li * R.st[R.ax_l]));
      tile[k][threadIdx.x & 31] = v;
    }
    __syncthreads();
    // store: threads along wavelength (the output's contiguous axis)
    for (int k = threadIdx.x >> 5; k < 32; k += blockDim.x >> 5) {
      const long long fi = f0 + k, li = l0 + (threadIdx.x & 31);
      if (fi < R.n[f] && li < R.nl) {
        long long c[4];
        c[f] = fi;
        c[g] = cg;
        c[h] = chh;
        c[R.ax_l] = li;
        const long long pixel = c[R.ax_col] * R.rows + c[R.ax_row];
        out[(pixel * 4 + c[R.ax_s]) * R.nl + li] = tile[threadIdx.x & 31][k];
      }
    }
    __syncthreads();
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
  if (roles != 15 || R.n[R.ax_s] != 4 || R.rows * info->ncols != info->npix || R.nl < 1)
    return pmh_fail(PM_EINVAL, "pm_fits_reorder: inconsistent cube description");
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const auto* in = static_cast<const unsigned int*>(data_dev);
  if (R.ax_l == 0) {
    long long blocks = (R.total + 255) / 256;
    if (blocks > (long long)sms * 16) blocks = (long long)sms * 16;
    reorder_direct<<<unsigned(blocks), 256, 0, s>>>(R, in, cube_dev);
  } else {
    // f: the input's contiguous axis (axis 0); g, h: the two other non-wavelength axes
    const int f = 0;
    int g = -1, h = -1;
    for (int a = 1; a < 4; ++a)
      if (a != R.ax_l) {
        if (g < 0) g = a;
        else h = a;
      }
    const long long work = ((R.n[f] + 31) / 32) * ((R.nl + 31) / 32) * R.n[g] * R.n[h];
    long long blocks = work < (long long)sms * 16 ? work : (long long)sms * 16;
    reorder_tiled<<<unsigned(blocks), 256, 0, s>>>(R, f, g, h, in, cube_dev);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char msg[160];
    std::snprintf(msg, sizeof msg, "pm_fits_reorder: %s", cudaGetErrorString(e));
    return pmh_fail(PM_EIO, msg);
  }
  return PM_OK;
}
