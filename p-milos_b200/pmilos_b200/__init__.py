"""pmilos_b200 -- Python host interface of libpmilos_b200.so (B200 ME inversion).

The compute path is the CUDA library behind the C ABI of ``include/pmilos.h``;
this module binds it with ctypes and mirrors the reference's per-run setup:

* ``LineData.from_lines_entry`` / ``line_from_quantum``  -- readFileCuanticLines +
  create_cuantic (readConfig.c:24-129, create_cuantic.c:24-294)
* ``grid_from_malla`` -- the wavelength grid of a .grid file (milos.c:176-196)
* ``psf_gaussian`` / ``psf_from_table`` -- fgauss_WL and the .psf route
  (fgauss.c:79-154; milos.c:266-344; milosUtils.c:684-738)
* ``Inverter.invert`` -- the per-pixel loop of milos.c:958-1009 (classical estimates,
  NaN fixes, lm_mils) over a whole batch
* ``Inverter.lm_mils`` -- one pixel, same contract as lm_mils (milosUtils.c:466-635)
* ``Inverter.synth`` -- mil_sinrf + me_der as the synthesis mode runs them

Buffers may be numpy arrays (host memory: the library stages them through the
GPU) or torch CUDA tensors (device memory: nothing is copied).  There is no CPU
fallback: without the built library or a B200 every compute call raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

from .files import (grid_from_malla, parse_lines_entry, read_grid_file, read_lines_file, read_model_file,
                    read_psf_file, read_trol_file)

__all__ = [
    "MODEL_FIELDS", "PmError", "LineData", "Inverter", "load_library", "line_from_quantum", "psf_gaussian",
    "psf_from_table", "grid_from_malla", "parse_lines_entry", "read_grid_file", "read_lines_file",
    "read_model_file", "read_psf_file", "read_trol_file", "PREC_FP64", "PREC_FP32", "SOLVE_DEFAULT",
    "SOLVE_EIGEN", "SOLVE_CHOLESKY", "SLIGHT_NONE", "SLIGHT_SHARED", "SLIGHT_PER_PIXEL", "Server", "Grid",
    "fits_header", "ingest_fits",
]

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(LIB_DIR, "libpmilos_b200.so")

MODEL_FIELDS = ("eta0", "B", "vlos", "dopp", "aa", "gm", "az", "S0", "S1", "mac", "alfa")
PREC_FP64, PREC_FP32 = 0, 1
SOLVE_DEFAULT, SOLVE_EIGEN, SOLVE_CHOLESKY = 0, 1, 2
SLIGHT_NONE, SLIGHT_SHARED, SLIGHT_PER_PIXEL = 0, 1, 2
MEM_HOST, MEM_DEVICE = 0, 1
PIX_CONVERGED, PIX_LAMBDA, PIX_MAXITER, PIX_NFREE, PIX_NONFINITE = 0, 1, 2, -1, -2
ZMAX = 16  # PM_ZEEMAN_MAX
NL_MAX = 128

# Every symbol include/pmilos.h declares (checked by the CPU test suite).
EXPORTED_SYMBOLS = (
    "pm_line_from_quantum", "pm_psf_gaussian", "pm_psf_interpolate", "pm_ctx_create", "pm_ctx_destroy",
    "pm_invert_batch", "pm_synth_batch", "pm_lm_mils", "pm_invert_batch_noalloc", "pm_get_stats", "pm_last_error",
    "pm_abi_version", "pm_get_tuning", "pm_set_tuning", "pm_autotune", "pm_server_create", "pm_server_submit",
    "pm_server_wait", "pm_server_get_stats", "pm_server_destroy", "pm_selftest_stalled_queue",
    "pm_fits_parse_header", "pm_fits_reorder", "pm_server_submit_device", "pm_invert_batch_grids",
    "pm_synth_batch_grids", "pm_server_set_slight",
)
SERVER_MAX_GRIDS = 4
SERVER_MAX_INFLIGHT = 256
ETIMEDOUT = -110
NOALLOC_MAX_PIXELS = 4096


class PmError(RuntimeError):
    """A negative return code of the C ABI (with pm_last_error's message)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class _Model(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in MODEL_FIELDS]


class _Line(ctypes.Structure):
    _fields_ = [
        ("lambda0", ctypes.c_double), ("n_pi", ctypes.c_int), ("n_sig", ctypes.c_int),
        ("nup", ctypes.c_double * ZMAX), ("nub", ctypes.c_double * ZMAX), ("nur", ctypes.c_double * ZMAX),
        ("wep", ctypes.c_double * ZMAX), ("web", ctypes.c_double * ZMAX), ("wer", ctypes.c_double * ZMAX),
        ("gl", ctypes.c_double), ("gu", ctypes.c_double), ("geff", ctypes.c_double), ("fo", ctypes.c_double),
    ]


class _Config(ctypes.Structure):
    _fields_ = [
        ("nlambda", ctypes.c_int), ("lambda_", ctypes.POINTER(ctypes.c_double)),
        ("psf", ctypes.POINTER(ctypes.c_double)), ("weight", ctypes.c_double * 4), ("noise", ctypes.c_double),
        ("ilambda", ctypes.c_double), ("toplim", ctypes.c_double), ("miter", ctypes.c_int),
        ("fix", ctypes.c_int * 11), ("nterms", ctypes.c_int), ("logclambda", ctypes.c_int),
        ("mu", ctypes.c_double), ("classical_estimates", ctypes.c_int), ("precision", ctypes.c_int),
        ("solver", ctypes.c_int),
    ]


class _Tuning(ctypes.Structure):
    _fields_ = [("variant", ctypes.c_int), ("staging_depth", ctypes.c_int), ("warps_per_block", ctypes.c_int),
                ("graphs", ctypes.c_int)]


class _FitsCube(ctypes.Structure):
    _fields_ = [("naxis", ctypes.c_int), ("naxes", ctypes.c_int64 * 4), ("axis_row", ctypes.c_int),
                ("axis_col", ctypes.c_int), ("axis_lambda", ctypes.c_int), ("axis_stokes", ctypes.c_int),
                ("from_ctype", ctypes.c_int), ("nrows", ctypes.c_int64), ("ncols", ctypes.c_int64),
                ("npix", ctypes.c_int64), ("nlambda", ctypes.c_int), ("data_offset", ctypes.c_int64),
                ("data_bytes", ctypes.c_int64)]


class _ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("max_inflight", ctypes.c_int), ("linger_ms", ctypes.c_double)]


class _ScanInfo(ctypes.Structure):
    _fields_ = [("npix", ctypes.c_int64), ("grid", ctypes.c_int), ("rc", ctypes.c_int), ("submit_ms", ctypes.c_double),
                ("admit_ms", ctypes.c_double), ("done_ms", ctypes.c_double), ("iterations", ctypes.c_int64)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("scans_done", ctypes.c_int64), ("pixels_done", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
                ("latency_p50_ms", ctypes.c_double), ("latency_p99_ms", ctypes.c_double),
                ("latency_max_ms", ctypes.c_double), ("busy_ms", ctypes.c_double),
                ("arena_peak_bytes", ctypes.c_size_t), ("prepass_launches", ctypes.c_int64)]


class _Stats(ctypes.Structure):
    _fields_ = [("pixels", ctypes.c_int64), ("iterations", ctypes.c_int64), ("accepted", ctypes.c_int64),
                ("eigen_fallbacks", ctypes.c_int64), ("kernel_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("graph_replays", ctypes.c_int64)]


_LIB = None


def load_library(path: str | None = None):
    """Load libpmilos_b200.so (raises if it has not been built: there is no fallback)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(f"{p} is missing: build it with __graft_entry__.build() (no CPU fallback exists)")
    L = ctypes.CDLL(p)
    vp, i64, D, F, I = ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_void_p
    L.pm_line_from_quantum.argtypes = [ctypes.c_double] * 7 + [ctypes.POINTER(_Line)]
    L.pm_psf_gaussian.argtypes = [ctypes.c_double, ctypes.c_int, D, D]
    L.pm_psf_interpolate.argtypes = [ctypes.c_int, D, D, ctypes.c_int, D, D]
    L.pm_ctx_create.argtypes = [ctypes.POINTER(_Line), ctypes.POINTER(_Config), vp, ctypes.POINTER(vp)]
    L.pm_ctx_destroy.argtypes = [vp]
    L.pm_invert_batch.argtypes = [vp, i64, F, F, ctypes.c_int, ctypes.POINTER(_Model), vp, vp, vp, vp, vp,
                                  ctypes.c_int]
    L.pm_synth_batch.argtypes = [vp, i64, vp, F, ctypes.c_int, vp, vp, ctypes.c_int]
    L.pm_invert_batch_grids.argtypes = [vp, i64, F, vp, F, ctypes.c_int, ctypes.POINTER(_Model), vp, vp, vp, vp, vp,
                                        ctypes.c_int]
    L.pm_synth_batch_grids.argtypes = [vp, i64, vp, vp, F, ctypes.c_int, vp, vp, ctypes.c_int]
    L.pm_lm_mils.argtypes = [vp, F, ctypes.POINTER(_Model), vp, ctypes.POINTER(ctypes.c_float), F,
                             ctypes.POINTER(ctypes.c_int)]
    L.pm_invert_batch_noalloc.argtypes = [ctypes.POINTER(_Line), ctypes.POINTER(_Config), i64, F, F, ctypes.c_int,
                                          ctypes.POINTER(_Model), vp, vp, vp, vp, vp, vp]
    L.pm_get_stats.argtypes = [vp, ctypes.POINTER(_Stats)]
    L.pm_get_tuning.argtypes = [vp, ctypes.POINTER(_Tuning)]
    L.pm_set_tuning.argtypes = [vp, ctypes.POINTER(_Tuning)]
    L.pm_autotune.argtypes = [vp, i64, F, F, ctypes.c_int, ctypes.POINTER(_Model), ctypes.c_int,
                              ctypes.POINTER(_Tuning)]
    L.pm_server_create.argtypes = [ctypes.POINTER(_Line), ctypes.POINTER(ctypes.POINTER(_Config)),
                                   ctypes.POINTER(_Model), ctypes.c_int, ctypes.POINTER(_ServerConfig),
                                   ctypes.POINTER(vp)]
    L.pm_server_submit.argtypes = [vp, ctypes.c_int, i64, F, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_uint64)]
    L.pm_server_submit_device.argtypes = [vp, ctypes.c_int, i64, F, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_uint64)]
    L.pm_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(_ScanInfo)]
    L.pm_server_set_slight.argtypes = [vp, ctypes.c_int, F, ctypes.c_int, i64]
    L.pm_server_get_stats.argtypes = [vp, ctypes.POINTER(_ServerStats)]
    L.pm_server_destroy.argtypes = [vp]
    L.pm_selftest_stalled_queue.argtypes = [vp, ctypes.c_double, ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_double)]
    L.pm_fits_parse_header.argtypes = [vp, ctypes.c_size_t, ctypes.POINTER(_FitsCube)]
    L.pm_fits_reorder.argtypes = [ctypes.POINTER(_FitsCube), vp, vp, vp]
    L.pm_last_error.restype = ctypes.c_char_p
    L.pm_abi_version.restype = ctypes.c_int
    if path is None:
        _LIB = L
    return L


def _check(rc: int) -> int:
    if rc < 0:
        raise PmError(rc, load_library().pm_last_error().decode())
    return rc


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@dataclass
class LineData:
    """Zeeman pattern + centre of one spectral line (what create_cuantic provides)."""

    lambda0: float
    quantum: tuple  # (SLOI, LLOI, JLOI, SUPI, LUPI, JUPI) as readFileCuanticLines decodes them
    _c: _Line = field(default=None, repr=False)

    def __post_init__(self):
        if self._c is None:
            self._c = _Line()
            _check(load_library().pm_line_from_quantum(self.lambda0, *[float(q) for q in self.quantum],
                                                       ctypes.byref(self._c)))

    @classmethod
    def from_lines_entry(cls, text: str, lambda0: float | None = None) -> "LineData":
        idx, lam, q = parse_lines_entry(text)
        return cls(lam if lambda0 is None else lambda0, q)

    @property
    def geff(self) -> float:
        return self._c.geff

    def cuantic_dat(self) -> np.ndarray:
        """The 7-double array readFileCuanticLines produces ({1, quantum numbers})."""
        return np.array([1.0, *self.quantum], dtype=np.float64)


def line_from_quantum(lambda0: float, sl, ll, jl, su, lu, ju) -> LineData:
    return LineData(lambda0, (sl, ll, jl, su, lu, ju))


def psf_gaussian(fwhm_ma: float, lam: np.ndarray) -> np.ndarray:
    lam = np.ascontiguousarray(lam, dtype=np.float64)
    out = np.zeros_like(lam)
    _check(load_library().pm_psf_gaussian(float(fwhm_ma), lam.size, _dptr(lam), _dptr(out)))
    return out


def psf_from_table(offsets_ma: np.ndarray, values: np.ndarray, grid_offsets_ma: np.ndarray) -> np.ndarray:
    dl = np.ascontiguousarray(offsets_ma, dtype=np.float64)
    ps = np.ascontiguousarray(values, dtype=np.float64)
    go = np.ascontiguousarray(grid_offsets_ma, dtype=np.float64)
    out = np.zeros_like(go)
    _check(load_library().pm_psf_interpolate(dl.size, _dptr(dl), _dptr(ps), go.size, _dptr(go), _dptr(out)))
    return out


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _model_struct(m) -> _Model:
    v = [float(x) for x in np.asarray(m, dtype=np.float64).ravel()]
    if len(v) != 11:
        raise ValueError("a model has 11 parameters (eta0, B, vlos, dopp, aa, gm, az, S0, S1, mac, alfa)")
    return _Model(*v)


class Inverter:
    """One pm_ctx: a wavelength grid, a line, a PSF and the control settings.

    Mirrors the inputs lm_mils takes from the control file (.mtrol): weights,
    noise (sigma^2 = 1/SN^2), initial diagonal element, toplim, number of cycles,
    the fix[] switches (reference order eta0, B, vlos, dopp, aa, gm, az, S0, S1,
    mac, alfa), NTERMS, the diagonal-acceleration switch and mu.  NTERMS
    defaults to 11 - !fix[10] - !fix[9] (milos.c:152-157 with a zero guess
    v_mac); give it explicitly (10 or 11) for guesses with v_mac fixed at a
    nonzero value.
    """

    def __init__(self, line: LineData, lam, psf=None, *, weights=(1.0, 1.0, 1.0, 1.0), noise=1e-6, ilambda=0.1,
                 toplim=1e-12, miter=50, fix=None, nterms=None, logclambda=0, mu=1.0, classical=True,
                 precision=PREC_FP32, solver=SOLVE_DEFAULT, stream=None):
        self.L = load_library()
        self.line = line
        self.lam = np.ascontiguousarray(lam, dtype=np.float64)
        self.nl = int(self.lam.size)
        self.psf = None if psf is None else np.ascontiguousarray(psf, dtype=np.float64)
        fix = list(fix) if fix is not None else [1] * 9 + [0, 0]
        if nterms is None:
            nterms = 11 - (0 if fix[10] else 1) - (0 if fix[9] else 1)
        self.nterms = nterms
        self.precision = precision
        c = _Config()
        c.nlambda = self.nl
        c.lambda_ = _dptr(self.lam)
        c.psf = _dptr(self.psf) if self.psf is not None else ctypes.POINTER(ctypes.c_double)()
        c.weight[:] = [float(w) for w in weights]
        c.noise, c.ilambda, c.toplim, c.miter = float(noise), float(ilambda), float(toplim), int(miter)
        c.fix[:] = [int(bool(f)) for f in fix]
        c.nterms, c.logclambda, c.mu = int(nterms), int(logclambda), float(mu)
        c.classical_estimates, c.precision, c.solver = int(bool(classical)), int(precision), int(solver)
        self._cfg = c
        ctx = ctypes.c_void_p()
        st = ctypes.c_void_p(int(stream)) if stream is not None else None
        _check(self.L.pm_ctx_create(ctypes.byref(line._c), ctypes.byref(c), st, ctypes.byref(ctx)))
        self.ctx = ctx

    def close(self):
        if getattr(self, "ctx", None):
            self.L.pm_ctx_destroy(self.ctx)
            self.ctx = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- batched inversion ----
    def invert(self, spectro, guess, *, slight=None, slight_mode=None, want_spectra=True, want_status=True,
               lam=None, out=None):
        """Invert [npix][4][nl] float32 profiles.  numpy in -> numpy out (host staging);
        torch CUDA in -> torch CUDA out (no copies).  lam: [npix][nl] absolute
        wavelengths of each pixel (pm_invert_batch_grids) instead of the grid.
        out (numpy input only): preallocated C-contiguous result arrays, a dict
        with "models" [npix][11] float64, "chisq" [npix] float32, "iters" [npix]
        int32 and, when wanted, "spectra" [npix][4][nl] float32 and "status" [npix]
        int32; in pinned, mapped host memory (e.g. torch's pin_memory) the kernel
        stores the results into them directly."""
        if _is_torch(spectro):
            if out is not None:
                raise ValueError("out= takes host arrays; device inputs return device tensors")
            return self._invert_device(spectro, guess, slight, slight_mode, want_spectra, want_status, lam)
        obs = np.ascontiguousarray(spectro, dtype=np.float32).reshape(-1, 4, self.nl)
        npix = obs.shape[0]
        lamp = None
        if lam is not None:
            lamp = np.ascontiguousarray(lam, dtype=np.float64)
            if lamp.size != npix * self.nl:
                raise ValueError("per-pixel wavelengths must be [npix][nl]")
        sl, mode = self._slight_host(slight, slight_mode, npix)
        shapes = {"models": ((npix, 11), np.float64), "chisq": ((npix,), np.float32), "iters": ((npix,), np.int32),
                  "spectra": ((npix, 4, self.nl), np.float32), "status": ((npix,), np.int32)}
        wanted = {"models": True, "chisq": True, "iters": True, "spectra": want_spectra, "status": want_status}
        arr = {}
        for k, (shape, dt) in shapes.items():
            if not wanted[k]:
                arr[k] = None
            elif out is not None and k in out:
                a = out[k]
                if not (isinstance(a, np.ndarray) and a.dtype == dt and a.shape == shape and a.flags.c_contiguous
                        and a.flags.writeable):
                    raise ValueError(f"out[{k!r}] must be a writeable C-contiguous {np.dtype(dt).name} array of "
                                     f"shape {shape}")
                arr[k] = a
            else:
                arr[k] = np.zeros(shape, dtype=dt)
        models, chi, its, sp, stt = (arr[k] for k in ("models", "chisq", "iters", "spectra", "status"))
        g = _model_struct(guess)
        outs = (ctypes.byref(g), models.ctypes.data, chi.ctypes.data, its.ctypes.data,
                None if sp is None else sp.ctypes.data, None if stt is None else stt.ctypes.data, MEM_HOST)
        slp = None if sl is None else sl.ctypes.data
        if lamp is None:
            _check(self.L.pm_invert_batch(self.ctx, npix, obs.ctypes.data, slp, mode, *outs))
        else:
            _check(self.L.pm_invert_batch_grids(self.ctx, npix, obs.ctypes.data, lamp.ctypes.data, slp, mode, *outs))
        out = {"models": models, "chisq": chi, "iters": its}
        if sp is not None:
            out["spectra"] = sp
        if stt is not None:
            out["status"] = stt
        return out

    def _slight_host(self, slight, mode, npix):
        if slight is None:
            return None, SLIGHT_NONE
        sl = np.ascontiguousarray(slight, dtype=np.float32)
        if mode is None:
            mode = SLIGHT_SHARED if sl.size == 4 * self.nl else SLIGHT_PER_PIXEL
        if mode == SLIGHT_PER_PIXEL and sl.size != npix * 4 * self.nl:
            raise ValueError("per-pixel stray light must be [npix][4][nl]")
        return sl, mode

    def _invert_device(self, spectro, guess, slight, slight_mode, want_spectra, want_status, lam=None):
        import torch

        obs = spectro.contiguous().view(-1, 4, self.nl)
        if obs.dtype != torch.float32 or not obs.is_cuda:
            raise TypeError("device inversion wants a float32 CUDA tensor")
        npix = obs.shape[0]
        dev = obs.device
        models = torch.empty((npix, 11), dtype=torch.float64, device=dev)
        chi = torch.empty(npix, dtype=torch.float32, device=dev)
        its = torch.empty(npix, dtype=torch.int32, device=dev)
        sp = torch.empty((npix, 4, self.nl), dtype=torch.float32, device=dev) if want_spectra else None
        stt = torch.empty(npix, dtype=torch.int32, device=dev) if want_status else None
        mode = SLIGHT_NONE
        slp = None
        if slight is not None:
            sl = slight.contiguous()
            mode = slight_mode if slight_mode is not None else (
                SLIGHT_SHARED if sl.numel() == 4 * self.nl else SLIGHT_PER_PIXEL)
            slp = sl.data_ptr()
        g = _model_struct(guess)
        outs = (ctypes.byref(g), models.data_ptr(), chi.data_ptr(), its.data_ptr(),
                None if sp is None else sp.data_ptr(), None if stt is None else stt.data_ptr(), MEM_DEVICE)
        if lam is None:
            _check(self.L.pm_invert_batch(self.ctx, npix, obs.data_ptr(), slp, mode, *outs))
        else:
            lamt = lam.contiguous()
            if lamt.dtype != torch.float64 or not lamt.is_cuda or lamt.numel() != npix * self.nl:
                raise TypeError("per-pixel wavelengths: a float64 CUDA tensor [npix][nl]")
            _check(self.L.pm_invert_batch_grids(self.ctx, npix, obs.data_ptr(), lamt.data_ptr(), slp, mode, *outs))
        out = {"models": models, "chisq": chi, "iters": its}
        if sp is not None:
            out["spectra"] = sp
        if stt is not None:
            out["status"] = stt
        return out

    # ---- forward synthesis ----
    def synth(self, models, *, slight=None, slight_mode=None, rf=False, lam=None):
        """Synthesize [npix][11] models -> [npix][4][nl] (+ RFs [npix][4][nterms][nl]).
        lam: [npix][nl] absolute wavelengths of each pixel (host arrays only)."""
        if _is_torch(models):
            import torch

            m = models.contiguous().to(torch.float64).view(-1, 11)
            npix = m.shape[0]
            sp = torch.empty((npix, 4, self.nl), dtype=torch.float32, device=m.device)
            rfo = torch.empty((npix, 4, self.nterms, self.nl), dtype=torch.float32, device=m.device) if rf else None
            mode, slp = SLIGHT_NONE, None
            if slight is not None:
                sl = slight.contiguous()
                mode = slight_mode if slight_mode is not None else (
                    SLIGHT_SHARED if sl.numel() == 4 * self.nl else SLIGHT_PER_PIXEL)
                slp = sl.data_ptr()
            _check(self.L.pm_synth_batch(self.ctx, npix, m.data_ptr(), slp, mode, sp.data_ptr(),
                                         None if rfo is None else rfo.data_ptr(), MEM_DEVICE))
            return (sp, rfo) if rf else sp
        m = np.ascontiguousarray(models, dtype=np.float64).reshape(-1, 11)
        npix = m.shape[0]
        sl, mode = self._slight_host(slight, slight_mode, npix)
        sp = np.zeros((npix, 4, self.nl), dtype=np.float32)
        rfo = np.zeros((npix, 4, self.nterms, self.nl), dtype=np.float32) if rf else None
        outs = (None if sl is None else sl.ctypes.data, mode, sp.ctypes.data,
                None if rfo is None else rfo.ctypes.data, MEM_HOST)
        if lam is None:
            _check(self.L.pm_synth_batch(self.ctx, npix, m.ctypes.data, *outs))
        else:
            lamp = np.ascontiguousarray(lam, dtype=np.float64)
            if lamp.size != npix * self.nl:
                raise ValueError("per-pixel wavelengths must be [npix][nl]")
            _check(self.L.pm_synth_batch_grids(self.ctx, npix, m.ctypes.data, lamp.ctypes.data, *outs))
        return (sp, rfo) if rf else sp

    # ---- lm_mils, batch of one ----
    def lm_mils(self, spectro, init_model, slight=None):
        """Returns (rc, model, spectra, chisq, iter) like lm_mils' outputs."""
        obs = np.ascontiguousarray(spectro, dtype=np.float32).reshape(4 * self.nl)
        m = _model_struct(init_model)
        sp = np.zeros(4 * self.nl, dtype=np.float32)
        chi = ctypes.c_float()
        it = ctypes.c_int()
        sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float32).reshape(4 * self.nl)
        rc = _check(self.L.pm_lm_mils(self.ctx, obs.ctypes.data, ctypes.byref(m), sp.ctypes.data, ctypes.byref(chi),
                                      None if sl is None else sl.ctypes.data, ctypes.byref(it)))
        model = np.array([getattr(m, n) for n in MODEL_FIELDS])
        return rc, model, sp.reshape(4, self.nl), chi.value, it.value

    def invert_noalloc(self, spectro, guess, *, slight=None, slight_mode=None, want_spectra=True, want_status=True):
        """The same inversion as ``invert`` on host arrays, through
        pm_invert_batch_noalloc: no GPU memory is allocated (the library stages
        through its built-in static device array), so at most
        NOALLOC_MAX_PIXELS pixels per call."""
        obs = np.ascontiguousarray(spectro, dtype=np.float32).reshape(-1, 4, self.nl)
        npix = obs.shape[0]
        sl, mode = self._slight_host(slight, slight_mode, npix)
        models = np.zeros((npix, 11), dtype=np.float64)
        chi = np.zeros(npix, dtype=np.float32)
        its = np.zeros(npix, dtype=np.int32)
        sp = np.zeros((npix, 4, self.nl), dtype=np.float32) if want_spectra else None
        stt = np.zeros(npix, dtype=np.int32) if want_status else None
        g = _model_struct(guess)
        _check(self.L.pm_invert_batch_noalloc(ctypes.byref(self.line._c), ctypes.byref(self._cfg), npix,
                                              obs.ctypes.data, None if sl is None else sl.ctypes.data, mode,
                                              ctypes.byref(g), models.ctypes.data, chi.ctypes.data, its.ctypes.data,
                                              None if sp is None else sp.ctypes.data,
                                              None if stt is None else stt.ctypes.data, None))
        out = {"models": models, "chisq": chi, "iters": its}
        if sp is not None:
            out["spectra"] = sp
        if stt is not None:
            out["status"] = stt
        return out

    @property
    def tuning(self) -> dict:
        t = _Tuning()
        _check(self.L.pm_get_tuning(self.ctx, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in _Tuning._fields_}

    @tuning.setter
    def tuning(self, value: dict):
        t = _Tuning()
        _check(self.L.pm_get_tuning(self.ctx, ctypes.byref(t)))
        for k, v in value.items():
            setattr(t, k, int(v))
        _check(self.L.pm_set_tuning(self.ctx, ctypes.byref(t)))

    def autotune(self, spectro, guess, *, slight=None, slight_mode=None, reps: int = 2) -> dict:
        """Time every candidate tuning on this host-memory sample and keep the fastest."""
        obs = np.ascontiguousarray(spectro, dtype=np.float32).reshape(-1, 4, self.nl)
        sl, mode = self._slight_host(slight, slight_mode, obs.shape[0])
        g = _model_struct(guess)
        t = _Tuning()
        _check(self.L.pm_autotune(self.ctx, obs.shape[0], obs.ctypes.data, None if sl is None else sl.ctypes.data,
                                  mode, ctypes.byref(g), int(reps), ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in _Tuning._fields_}

    def selftest_stalled_queue(self, limit_ms: float = 50.0) -> tuple[int, float]:
        """Launch the streamed kernel on a queue nothing publishes to: returns
        (queue error word, kernel ms); 1 = the bounded wait gave up by itself."""
        err = ctypes.c_int()
        ms = ctypes.c_double()
        _check(self.L.pm_selftest_stalled_queue(self.ctx, float(limit_ms), ctypes.byref(err), ctypes.byref(ms)))
        return err.value, ms.value

    def stats(self) -> dict:
        s = _Stats()
        _check(self.L.pm_get_stats(self.ctx, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in _Stats._fields_}


# ---- serving ----
@dataclass
class Grid:
    """One wavelength grid a Server holds resident: the pm_config fields of an
    Inverter plus the initial model of the grid's scans."""
    lam: np.ndarray
    psf: np.ndarray | None = None
    guess: np.ndarray | None = None
    weights: tuple = (1.0, 1.0, 1.0, 1.0)
    noise: float = 1e-6
    ilambda: float = 0.1
    toplim: float = 1e-12
    miter: int = 50
    fix: list | None = None
    nterms: int | None = None
    mu: float = 1.0
    classical: bool = True
    precision: int = PREC_FP32
    solver: int = SOLVE_DEFAULT


class Server:
    """pm_server: continuous batching of spectral scans on resident grids.

    submit() queues a scan (a [npix][4][nl] float32 host array; pinned memory
    lets its copy overlap the kernel) and returns its id at once; wait() blocks
    until its models, chi^2, iterations and status are in host memory.  Scans
    that arrive while others are on the GPU join the running kernel as device
    memory (hbm_budget_bytes) and in-flight slots free up."""

    def __init__(self, line: LineData, grids, *, hbm_budget_bytes: int = 8 << 30, max_inflight: int = 64,
                 linger_ms: float = 2.0):
        self.L = load_library()
        self.line = line
        self.grids = list(grids)
        self._keep = []
        cfgs = (ctypes.POINTER(_Config) * len(self.grids))()
        guesses = (_Model * len(self.grids))()
        self.nl = []
        for i, g in enumerate(self.grids):
            lam = np.ascontiguousarray(g.lam, dtype=np.float64)
            psf = None if g.psf is None else np.ascontiguousarray(g.psf, dtype=np.float64)
            fix = list(g.fix) if g.fix is not None else [1] * 9 + [0, 0]
            gmac = 0.0 if g.guess is None else float(np.asarray(g.guess, dtype=np.float64)[9])
            nterms = g.nterms if g.nterms is not None else \
                11 - (0 if fix[10] else 1) - (0 if (fix[9] or gmac != 0.0) else 1)
            c = _Config()
            c.nlambda = lam.size
            c.lambda_ = _dptr(lam)
            c.psf = _dptr(psf) if psf is not None else ctypes.POINTER(ctypes.c_double)()
            c.weight[:] = [float(w) for w in g.weights]
            c.noise, c.ilambda, c.toplim, c.miter = float(g.noise), float(g.ilambda), float(g.toplim), int(g.miter)
            c.fix[:] = [int(bool(f)) for f in fix]
            c.nterms, c.logclambda, c.mu = int(nterms), 0, float(g.mu)
            c.classical_estimates, c.precision, c.solver = int(bool(g.classical)), int(g.precision), int(g.solver)
            self._keep += [lam, psf, c]
            cfgs[i] = ctypes.pointer(c)
            guesses[i] = _model_struct(g.guess if g.guess is not None else np.array(
                [8.0, 400.0, 0.0, 0.03, 0.1, 30.0, 30.0, 0.25, 0.75, 0.0, 1.0]))
            self.nl.append(int(lam.size))
        sc = _ServerConfig(int(hbm_budget_bytes), int(max_inflight), float(linger_ms))
        srv = ctypes.c_void_p()
        _check(self.L.pm_server_create(ctypes.byref(line._c), cfgs, guesses, len(self.grids), ctypes.byref(sc),
                                       ctypes.byref(srv)))
        self.srv = srv
        self._pending = {}

    def set_slight(self, grid: int, slight) -> None:
        """Stray light of a grid, before the first submit (pm_server_set_slight):
        a [4][nl] profile for every pixel, a [npix][4][nl] cube (then every scan
        on the grid has npix pixels, in the cube's pixel order), or None."""
        if slight is None:
            _check(self.L.pm_server_set_slight(self.srv, int(grid), None, SLIGHT_NONE, 0))
            return
        sl = np.ascontiguousarray(slight, dtype=np.float32)
        nl = self.nl[grid]
        if sl.size == 4 * nl:
            mode, npix = SLIGHT_SHARED, 1
        else:
            sl = sl.reshape(-1, 4, nl)
            mode, npix = SLIGHT_PER_PIXEL, sl.shape[0]
        _check(self.L.pm_server_set_slight(self.srv, int(grid), sl.ctypes.data, mode, npix))

    def submit(self, grid: int, spectro, want_status: bool = True) -> int:
        """Queue a scan: a host array, or a CUDA float32 tensor already on this GPU
        (used in place; keep it unchanged until the scan is done)."""
        if not 0 <= grid < len(self.nl):
            raise PmError(-22, f"no grid {grid} (the server holds {len(self.nl)})")
        nl = self.nl[grid]
        on_device = _is_torch(spectro) and spectro.is_cuda
        if on_device:
            import torch

            if spectro.dtype != torch.float32 or not spectro.is_contiguous():
                raise TypeError("a device scan must be a contiguous float32 CUDA tensor")
            obs, size, ptr = spectro, spectro.numel(), spectro.data_ptr()
        else:
            obs = spectro if (isinstance(spectro, np.ndarray) and spectro.dtype == np.float32 and
                              spectro.flags.c_contiguous) else np.ascontiguousarray(spectro, dtype=np.float32)
            size, ptr = obs.size, obs.ctypes.data
        if size % (4 * nl):
            raise ValueError(f"grid {grid} has {nl} wavelengths: spectro must be [npix][4][{nl}]")
        npix = size // (4 * nl)
        models = np.zeros((npix, 11))
        chi = np.zeros(npix, dtype=np.float32)
        its = np.zeros(npix, dtype=np.int32)
        stt = np.zeros(npix, dtype=np.int32) if want_status else None
        sid = ctypes.c_uint64()
        fn = self.L.pm_server_submit_device if on_device else self.L.pm_server_submit
        _check(fn(self.srv, int(grid), npix, ptr, models.ctypes.data, chi.ctypes.data, its.ctypes.data,
                  None if stt is None else stt.ctypes.data, ctypes.byref(sid)))
        self._pending[sid.value] = (obs, models, chi, its, stt)
        return sid.value

    def wait(self, sid: int, timeout: float = 600.0) -> dict:
        info = _ScanInfo()
        rc = self.L.pm_server_wait(self.srv, ctypes.c_uint64(sid), float(timeout), ctypes.byref(info))
        if rc == ETIMEDOUT:
            raise TimeoutError(f"scan {sid} not done after {timeout} s")
        bufs = self._pending.pop(sid, None)
        _check(rc)
        _, models, chi, its, stt = bufs
        out = {"models": models, "chisq": chi, "iters": its,
               "info": {k: getattr(info, k) for k, _ in _ScanInfo._fields_}}
        if stt is not None:
            out["status"] = stt
        return out

    def stats(self) -> dict:
        st = _ServerStats()
        _check(self.L.pm_server_get_stats(self.srv, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _ServerStats._fields_}

    def close(self):
        if getattr(self, "srv", None):
            self.L.pm_server_destroy(self.srv)
            self.srv = None
            self._pending.clear()

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---- cube ingest ----
def _fits_struct(raw) -> "_FitsCube":
    buf = np.frombuffer(raw, dtype=np.uint8) if not isinstance(raw, np.ndarray) else raw.view(np.uint8).ravel()
    info = _FitsCube()
    _check(load_library().pm_fits_parse_header(buf.ctypes.data, buf.size, ctypes.byref(info)))
    return info


def fits_header(raw) -> dict:
    """Parse a FITS spectro cube's primary header (bytes of the file, at least up
    to END): axis sizes, the axis of each role, pixels, wavelengths, data block."""
    info = _fits_struct(raw)
    out = {k: getattr(info, k) for k, _ in _FitsCube._fields_}
    out["naxes"] = list(info.naxes)
    return out


def ingest_fits(source, stream=None):
    """A FITS spectro cube (a path or the file's bytes) as a CUDA float32 tensor
    [npix][4][nlambda]: the data block is copied to the device as stored and
    reordered there by pm_fits_reorder."""
    import torch

    raw = np.fromfile(source, dtype=np.uint8) if isinstance(source, (str, os.PathLike)) else \
        np.frombuffer(source, dtype=np.uint8)
    info = _fits_struct(raw)
    o, n = int(info.data_offset), int(info.data_bytes)
    if raw.size < o + n:
        raise PmError(-22, f"the FITS data block needs {o + n} bytes, the file has {raw.size}")
    data = torch.from_numpy(np.array(raw[o:o + n], copy=True)).to("cuda", non_blocking=False)
    cube = torch.empty((int(info.npix), 4, int(info.nlambda)), dtype=torch.float32, device="cuda")
    st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    _check(load_library().pm_fits_reorder(ctypes.byref(info), data.data_ptr(), cube.data_ptr(), ctypes.c_void_p(st)))
    torch.cuda.current_stream().synchronize() if stream is None else None
    return cube
