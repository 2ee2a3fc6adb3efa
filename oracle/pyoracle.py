"""ctypes bindings for the oracle libraries (TEST INFRASTRUCTURE ONLY).

Two libraries share one calling convention:

* ``Restatement`` -- this project's C restatement (oracle/pm_oracle.c), built into
  ``oracle/build/libpmoracle_{f32,f64}.so``.  This is the oracle the GPU tests
  check against; it builds anywhere gcc exists.
* ``Reference`` -- the reference's own hot-path sources compiled unmodified
  against project shims (oracle/ref_harness.c), built into
  ``oracle/_ref/libpmref_{f32,f64}[_fast].so``.  It exists only where the
  reference tree was available at build time; it pins the restatement.

Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline leg of bench.py may
import this module.  The product path never does.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "build")
REF = os.path.join(HERE, "_ref")

_D = ctypes.POINTER(ctypes.c_double)
_F = ctypes.POINTER(ctypes.c_float)
_I = ctypes.POINTER(ctypes.c_int)


def _d(a):
    return None if a is None else a.ctypes.data_as(_D)


def _f(a):
    return None if a is None else a.ctypes.data_as(_F)


def _i(a):
    return None if a is None else a.ctypes.data_as(_I)


def build(quiet: bool = True, refsrc: str | None = None) -> None:
    """Compile the restatement (always) and the reference, from its src/
    directory given as ``refsrc`` or $PM_REFERENCE_SRC (skipped when neither
    names an existing directory)."""
    import subprocess

    targets = ["own"]
    refsrc = refsrc or os.environ.get("PM_REFERENCE_SRC")
    if refsrc and os.path.isdir(refsrc):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, f"REFSRC={refsrc or ''}", *targets], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def reference_available(flavour: str = "f64") -> bool:
    return os.path.exists(os.path.join(REF, f"libpmref_{flavour}.so"))


@dataclass
class LineSetup:
    """Spectral line + wavelength grid + PSF, the per-run constants of lm_mils."""

    lam: np.ndarray          # absolute wavelengths [A], float64 (nl,)
    lambda0: float           # line centre [A]
    cuantic: np.ndarray      # [1, SLOI, LLOI, JLOI, SUPI, LUPI, JUPI]
    psf: np.ndarray | None   # nl taps centred at nl//2, or None
    nterms: int

    @property
    def nl(self) -> int:
        return int(self.lam.shape[0])


class _Lib:
    """Common wrapper; subclasses bind either the pmo_* or the pmref_* symbols."""

    real_bytes: int

    def synth(self, model, slight=None, mu=1.0, fix=None, rf=True):
        nl, K = self.setup.nl, self.setup.nterms
        m = np.ascontiguousarray(model, dtype=np.float64)
        sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float64).ravel()
        fx = np.ascontiguousarray(fix if fix is not None else [1] * 11, dtype=np.int32)
        sp = np.zeros(4 * nl)
        ds = np.zeros(4 * nl * K) if rf else None
        rc = self._synth(m, sl, mu, fx, sp, ds)
        if rc != 0:
            raise RuntimeError(f"synth failed rc={rc}")
        return sp.reshape(4, nl), (None if ds is None else ds.reshape(4, K, nl))

    def classical(self, spectro, guess, initial_use=True):
        """estimacionesClasicas on one pixel from guess: initial_use=True as
        before lm_mils, False as the classical-estimates-only mode."""
        m = np.ascontiguousarray(guess, dtype=np.float64).copy()
        self._classical(np.ascontiguousarray(spectro, dtype=np.float32).ravel(), m, initial_use)
        return m

    def invert(self, spectro, guess, *, slight=None, slight_per_pixel=False, classical=True, miter=50,
               weights=(1.0, 1.0, 1.0, 1.0), noise=1e-6, ilambda=0.1, logclambda=0, toplim=1e-12, mu=1.0,
               fix=None, want_spectra=True):
        """Invert [npix][4][nl] float32 profiles; returns a dict of numpy arrays."""
        nl = self.setup.nl
        obs = np.ascontiguousarray(spectro, dtype=np.float32).reshape(-1, 4 * nl)
        npix = obs.shape[0]
        g = np.ascontiguousarray(guess, dtype=np.float64)
        sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float64).ravel()
        w = np.ascontiguousarray(weights, dtype=np.float64)
        fx = np.ascontiguousarray(fix if fix is not None else [1] * 9 + [0, 0], dtype=np.int32)
        models = np.zeros((npix, 11))
        chi = np.zeros(npix, dtype=np.float32)
        its = np.zeros(npix, dtype=np.int32)
        acc = np.zeros(npix, dtype=np.int32)
        st = np.full(npix, -9, dtype=np.int32)
        sp = np.zeros((npix, 4 * nl), dtype=np.float32) if want_spectra else None
        self._batch(npix, obs, g, sl, int(slight_per_pixel), int(classical), miter, w, noise, ilambda,
                    logclambda, toplim, mu, fx, models, chi, its, sp, acc, st)
        out = {"models": models, "chisq": chi, "iters": its, "accepted": acc}
        if (st != -9).all():  # the restatement reports how each pixel's loop ended (PM_PIX_* codes)
            out["status"] = st
        if sp is not None:
            out["spectra"] = sp.reshape(npix, 4, nl)
        return out


class Restatement(_Lib):
    def __init__(self, setup: LineSetup, flavour: str = "f64"):
        path = os.path.join(BUILD, f"libpmoracle_{flavour}.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.pmo_create.restype = ctypes.c_void_p
        L.pmo_create.argtypes = [ctypes.c_int, _D, ctypes.c_double, _D, _D, ctypes.c_int]
        L.pmo_destroy.argtypes = [ctypes.c_void_p]
        L.pmo_synth.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_double, _I, _D, _D]
        L.pmo_classical.argtypes = [ctypes.c_void_p, _F, _D]
        L.pmo_classical_only.argtypes = [ctypes.c_void_p, _F, _D]
        L.pmo_invert_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, _F, _D, _D, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, _D, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_double, _I, _D, _F, _I, _F, _I, _I]
        L.pmo_fvoigt.argtypes = [ctypes.c_double, _D, ctypes.c_int, _D, _D]
        L.pmo_conv.argtypes = [ctypes.c_void_p, _D, ctypes.c_int, ctypes.c_double]
        L.pmo_svd_solve.argtypes = [ctypes.c_int, _D, _D, _D]
        L.pmo_cuantic.argtypes = [ctypes.c_void_p, _D, ctypes.c_int]
        self.L = L
        self.setup = setup
        self.real_bytes = L.pmo_sizeof_real()
        lam = np.ascontiguousarray(setup.lam, dtype=np.float64)
        cq = np.ascontiguousarray(setup.cuantic, dtype=np.float64)
        psf = None if setup.psf is None else np.ascontiguousarray(setup.psf, dtype=np.float64)
        self.ctx = L.pmo_create(setup.nl, _d(lam), setup.lambda0, _d(cq), _d(psf), setup.nterms)
        if not self.ctx:
            raise RuntimeError("pmo_create failed")

    def __del__(self):
        if getattr(self, "ctx", None):
            self.L.pmo_destroy(self.ctx)
            self.ctx = None

    def _synth(self, m, sl, mu, fx, sp, ds):
        return self.L.pmo_synth(self.ctx, _d(m), _d(sl), mu, _i(fx), _d(sp), _d(ds))

    def _classical(self, obs, m, initial_use=True):
        (self.L.pmo_classical if initial_use else self.L.pmo_classical_only)(self.ctx, _f(obs), _d(m))

    def _batch(self, npix, obs, g, sl, slpp, cl, miter, w, noise, ilam, logc, toplim, mu, fx, models, chi, its,
               sp, acc, st):
        self.L.pmo_invert_batch(self.ctx, npix, _f(obs), _d(g), _d(sl), slpp, cl, miter, _d(w), noise, ilam, logc,
                                toplim, mu, _i(fx), _d(models), _f(chi), _i(its), _f(sp), _i(acc), _i(st))

    def fvoigt(self, damp, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        h = np.zeros_like(v)
        f = np.zeros_like(v)
        self.L.pmo_fvoigt(damp, _d(v), v.size, _d(h), _d(f))
        return h, f

    def conv(self, x, mode, ic=0.0):
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        self.L.pmo_conv(self.ctx, _d(x), mode, ic)
        return x

    def svd_solve(self, covar, beta):
        K = len(beta)
        h = np.ascontiguousarray(covar, dtype=np.float64).copy()
        b = np.ascontiguousarray(beta, dtype=np.float64)
        d = np.zeros(K)
        self.L.pmo_svd_solve(K, _d(h), _d(b), _d(d))
        return d

    def cuantic(self):
        out = np.zeros(128)
        n = self.L.pmo_cuantic(self.ctx, _d(out), 128)
        return out[:n]


class Reference(_Lib):
    """The reference's own sources (single global state: one instance at a time)."""

    def __init__(self, setup: LineSetup, flavour: str = "f64"):
        path = os.path.join(REF, f"libpmref_{flavour}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        L.pmref_setup.argtypes = [ctypes.c_int, _D, ctypes.c_double, _D, _D, ctypes.c_int]
        L.pmref_synth.argtypes = [_D, _D, ctypes.c_double, _I, _D, _D]
        L.pmref_classical.argtypes = [_F, _D]
        L.pmref_classical_only.argtypes = [_F, _D]
        L.pmref_invert_batch.argtypes = [ctypes.c_int, _F, _D, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, _I, _D, _F, _I, _F]
        L.pmref_fvoigt.argtypes = [ctypes.c_double, _D, ctypes.c_int, _D, _D]
        L.pmref_conv.argtypes = [_D, ctypes.c_int, _D, ctypes.c_int, ctypes.c_double]
        L.pmref_svd_solve.argtypes = [_D, _D, _D]
        L.pmref_cuantic.argtypes = [_D, ctypes.c_int]
        L.pmref_fgauss_wl.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, _D]
        L.pmref_interp_psf.argtypes = [_D, _D, ctypes.c_int, _D, ctypes.c_int, ctypes.c_double, _D]
        self.L = L
        self.setup = setup
        self.real_bytes = L.pmref_sizeof_real()
        lam = np.ascontiguousarray(setup.lam, dtype=np.float64)
        cq = np.ascontiguousarray(setup.cuantic, dtype=np.float64)
        self._psf = None if setup.psf is None else np.ascontiguousarray(setup.psf, dtype=np.float64)
        rc = L.pmref_setup(setup.nl, _d(lam), setup.lambda0, _d(cq), _d(self._psf), setup.nterms)
        if rc != 0:
            raise RuntimeError("pmref_setup failed")

    def _synth(self, m, sl, mu, fx, sp, ds):
        return self.L.pmref_synth(_d(m), _d(sl), mu, _i(fx), _d(sp), _d(ds))

    def _classical(self, obs, m, initial_use=True):
        (self.L.pmref_classical if initial_use else self.L.pmref_classical_only)(_f(obs), _d(m))

    def _batch(self, npix, obs, g, sl, slpp, cl, miter, w, noise, ilam, logc, toplim, mu, fx, models, chi, its,
               sp, acc, st):
        acc[:] = -1  # the reference does not count accepted steps nor report how its loop ended
        self.L.pmref_invert_batch(npix, _f(obs), _d(g), _d(sl), slpp, cl, miter, _d(w), noise, ilam, logc, toplim,
                                  mu, _i(fx), _d(models), _f(chi), _i(its), _f(sp))

    def fvoigt(self, damp, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        h = np.zeros_like(v)
        f = np.zeros_like(v)
        rc = self.L.pmref_fvoigt(damp, _d(v), v.size, _d(h), _d(f))
        if rc != 0:
            raise ValueError("fvoigt: at most nl points per call")
        return h, f

    def conv(self, x, mode, ic=0.0):
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        self.L.pmref_conv(_d(x), x.size, self._psf, mode, ic)
        return x

    def svd_solve(self, covar, beta):
        K = len(beta)
        h = np.ascontiguousarray(covar, dtype=np.float64).copy()
        b = np.ascontiguousarray(beta, dtype=np.float64)
        d = np.zeros(K)
        self.L.pmref_svd_solve(_d(h), _d(b), _d(d))
        return d

    def cuantic(self):
        out = np.zeros(128)
        n = self.L.pmref_cuantic(_d(out), 128)
        return out[:n]

    def fgauss_wl(self, fwhm_ma, step, lambda_first, lambda_central, n):
        out = np.zeros(n)
        self.L.pmref_fgauss_wl(fwhm_ma, step, lambda_first, lambda_central, n, _d(out))
        return out

    def interp_psf(self, dl, psf, offsets, offset):
        dl = np.ascontiguousarray(dl, dtype=np.float64)
        psf = np.ascontiguousarray(psf, dtype=np.float64)
        offs = np.ascontiguousarray(offsets, dtype=np.float64)
        out = np.zeros(offs.size)
        self.L.pmref_interp_psf(_d(dl), _d(psf), dl.size, _d(offs), offs.size, offset, _d(out))
        return out


# ---- cube ingest ----
def fits_bytes(data: np.ndarray, ctypes_: list | None) -> bytes:
    """A FITS file (primary HDU, BITPIX = -32) holding ``data``, a float32 array
    whose numpy shape is (NAXIS4, NAXIS3, NAXIS2, NAXIS1); ``ctypes_``: CTYPE1..4
    strings, or None for a header without them."""
    dims = list(data.shape[::-1])
    cards = ["SIMPLE  =                    T", "BITPIX  =                  -32", "NAXIS   =                    4"]
    cards += [f"NAXIS{i + 1}  = {d:20d}" for i, d in enumerate(dims)]
    if ctypes_:
        cards += [f"CTYPE{i + 1}  = '{c:<8s}'" for i, c in enumerate(ctypes_)]
    cards.append("END")
    hdr = "".join(c.ljust(80) for c in cards).encode("ascii")
    hdr += b" " * (-len(hdr) % 2880)
    body = np.ascontiguousarray(data, dtype=">f4").tobytes()
    body += b"\0" * (-len(body) % 2880)
    return hdr + body


def fits_roles(dims: list, ctypes_: list | None) -> tuple:
    """(row, col, lambda, stokes) axis indices as readFitsSpectroImage assigns
    them (utilsFits.c:69-150): from CTYPE1..4, else smallest axis = Stokes, the
    smallest other = wavelength, the remaining two rows then columns."""
    if ctypes_:
        idx = {c.strip(): i for i, c in enumerate(ctypes_)}
        return idx["HPLN-TAN"], idx["HPLT-TAN"], idx["WAVE-GRI"], idx["STOKES"]
    s = min(range(4), key=lambda a: (dims[a], a))
    lam = min((a for a in range(4) if a != s), key=lambda a: (dims[a], a))
    rest = [a for a in range(4) if a not in (s, lam)]
    return rest[0], rest[1], lam, s


def fits_ingest(data: np.ndarray, ctypes_: list | None) -> np.ndarray:
    """Restatement of the generic reorder (utilsFits.c:242-336): out[pixel][s][l]
    with pixel = col * rows + row, for an array of numpy shape
    (NAXIS4, NAXIS3, NAXIS2, NAXIS1)."""
    dims = list(data.shape[::-1])
    row, col, lam, s = fits_roles(dims, ctypes_)
    f = np.asarray(data, dtype=np.float32)
    # numpy axis of FITS axis a is 3 - a; target order (col, row, stokes, lambda)
    t = np.transpose(f, (3 - col, 3 - row, 3 - s, 3 - lam))
    return np.ascontiguousarray(t).reshape(dims[col] * dims[row], dims[s], dims[lam])


def reference_fits_read(path: str, nlambda: int, npix_cap: int):
    """The reference's own reader (oracle/_ref/libpmref_fits.so): (cube, rows, cols)."""
    lib = ctypes.CDLL(os.path.join(REF, "libpmref_fits.so"))
    lib.pmref_fits_read.argtypes = [ctypes.c_char_p, ctypes.c_int, _F, ctypes.c_longlong, _I, _I]
    out = np.zeros(npix_cap * 4 * nlambda, dtype=np.float32)
    rows, cols = ctypes.c_int(), ctypes.c_int()
    rc = lib.pmref_fits_read(path.encode(), nlambda, _f(out), out.size, ctypes.byref(rows), ctypes.byref(cols))
    if rc != 0:
        raise RuntimeError(f"reference reader failed ({rc})")
    n = rows.value * cols.value
    return out[: n * 4 * nlambda].reshape(n, 4, nlambda), rows.value, cols.value


def reference_fits_straylight(path: str, cap: int = 1 << 20):
    """readFitsStrayLightFile (oracle/_ref/libpmref_fits.so): (array, nl, ns, nx, ny)."""
    lib = ctypes.CDLL(os.path.join(REF, "libpmref_fits.so"))
    lib.pmref_fits_straylight.argtypes = [ctypes.c_char_p, _F, ctypes.c_longlong, _I, _I, _I, _I]
    out = np.zeros(cap, dtype=np.float32)
    nl, ns, nx, ny = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rc = lib.pmref_fits_straylight(path.encode(), _f(out), out.size, ctypes.byref(nl), ctypes.byref(ns),
                                   ctypes.byref(nx), ctypes.byref(ny))
    if rc != 0:
        raise RuntimeError(f"reference stray-light reader failed ({rc})")
    n = nl.value * ns.value * (nx.value * ny.value if nx.value and ny.value else 1)
    return out[:n].copy(), nl.value, ns.value, nx.value, ny.value


def reference_fits_lambda(path: str, cap: int = 4096):
    """readFitsLambdaToArray on a 2-D wavelength file: (index_line, lambda)."""
    lib = ctypes.CDLL(os.path.join(REF, "libpmref_fits.so"))
    lib.pmref_fits_lambda.argtypes = [ctypes.c_char_p, _D, ctypes.c_int, _I, _I]
    out = np.zeros(cap)
    idx, nl = ctypes.c_int(), ctypes.c_int()
    rc = lib.pmref_fits_lambda(path.encode(), _d(out), cap, ctypes.byref(idx), ctypes.byref(nl))
    if rc != 0:
        raise RuntimeError(f"reference wavelength reader failed ({rc})")
    return idx.value, out[:nl.value].copy()
