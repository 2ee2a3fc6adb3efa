"""Readers for the reference's text inputs (host logic only; no GPU).

Each function restates one reader of readConfig.c / milos.c so that a user of the
reference can point this library at the same files:

* ``parse_lines_entry`` / ``read_lines_file`` -- readFileCuanticLines (readConfig.c:24-129)
* ``read_grid_file`` + ``grid_from_malla``      -- readMallaGrid (readConfig.c:295-335) and the
  grid construction of milos.c:176-196
* ``read_psf_file``                             -- readPSFFile (readConfig.c:341-365)
* ``read_model_file``                           -- readInitialModel (readConfig.c:136-191)
* ``read_trol_file``                            -- readTrolFile (readConfig.c:420-1023), the
  42 positional lines of a .mtrol file
* ``read_stray_light_fits``                     -- readFitsStrayLightFile (utilsFits.c:881-1199)
* ``read_wavelength_fits``                      -- readFitsLambdaToArray (utilsFits.c:749-833)
"""
from __future__ import annotations

import math
import os
import re

import numpy as np

from .specs import grid_from_malla  # noqa: F401  (the .grid rules, milos.c:176-196)

# readFileCuanticLines' letters (readConfig.c:46-95, J for L = 6 as it has it),
# and the spectroscopic I and K it leaves undecoded (L unset there)
_LEVELS = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5, "J": 6, "I": 6, "K": 7}
_LINE_RE = re.compile(
    r"^\s*(\d+)=(\S+)\s+(\d+)\s+([-+0-9.eE]+)\s+([-+0-9.eE]+)\s+([-+0-9.eE]+)\s+-([0-9.eE+-]+)\s+"
    r"(\d+)([A-Za-z])\s*([0-9.]+)-\s*(\d+)([A-Za-z])\s*([0-9.]+)")


def parse_lines_entry(text: str):
    """One LINES entry -> (index, lambda0 [A], (SLOI, LLOI, JLOI, SUPI, LUPI, JUPI)).

    Multiplicities 2S+1 are turned into spins (S = (2S+1 - 1) / 2, integer
    division as in the reference) and level letters into L."""
    m = _LINE_RE.match(text)
    if not m:
        raise ValueError(f"not a LINES entry: {text!r}")
    idx = int(m.group(1))
    lam = float(m.group(4))
    sl = (int(m.group(8)) - 1) // 2
    ll = _LEVELS.get(m.group(9).upper())
    jl = float(m.group(10))
    su = (int(m.group(11)) - 1) // 2
    lu = _LEVELS.get(m.group(12).upper())
    ju = float(m.group(13))
    if ll is None or lu is None:
        raise ValueError(f"unknown term letter in {text!r}")
    return idx, lam, (float(sl), float(ll), jl, float(su), float(lu), ju)


def read_lines_file(path: str, index: int):
    """The entry with the given index from a LINES file (readFileCuanticLines)."""
    with open(path) as f:
        for line in f:
            try:
                idx, lam, q = parse_lines_entry(line)
            except ValueError:
                continue
            if idx == index:
                return lam, q
    raise KeyError(f"line {index} not in {path}")


def read_grid_file(path: str):
    """(line index, initial, step, final) in mA from a .grid file (readMallaGrid)."""
    found = False
    with open(path) as f:
        for line in f:
            if found:
                m = re.match(r"\s*(\d+)[^:]*:\s*([-+0-9.eE]+)\s*,\s*([-+0-9.eE]+)\s*,\s*([-+0-9.eE]+)", line)
                if not m:
                    raise ValueError(f"bad grid line in {path}: {line!r}")
                return int(m.group(1)), float(m.group(2)), float(m.group(3)), float(m.group(4))
            if line.startswith("------"):
                found = True
    raise ValueError(f"no grid definition in {path}")


def read_psf_file(path: str):
    """(offsets [mA], values) of a two-column .psf file (readPSFFile)."""
    d = np.loadtxt(path, ndmin=2)
    return np.ascontiguousarray(d[:, 0]), np.ascontiguousarray(d[:, 1])


_MODEL_KEYS = (("magnetic field", 1), ("gamma", 5), ("phi", 6), ("eta_0", 0), ("Doppler width", 3),
               ("damping", 4), ("filling factor", 10), ("v_mac", 9), ("LOS velocity", 2), ("S_0", 7), ("S_1", 8))


def read_model_file(path: str) -> np.ndarray:
    """11 model parameters from a .mod file (readInitialModel); unset entries are 0."""
    m = np.zeros(11)
    with open(path) as f:
        for line in f:
            if ":" not in line:
                continue
            name, rest = line.split(":", 1)
            try:
                val = float(rest.split("!")[0].split()[0])
            except (ValueError, IndexError):
                continue
            for key, idx in _MODEL_KEYS:
                if key in name:
                    m[idx] = val
    return m


def _field(line: str):
    if ":" not in line:
        return ""
    return line.split(":", 1)[1].split("!")[0].strip()


def read_trol_file(path: str) -> dict:
    """The fields of a .mtrol control file that the inversion uses (readTrolFile).

    Blank fields keep the defaults of loadInitialValues (readConfig.c:371-408):
    weights 1, noise 1e-6, initial diagonal 0.1, toplim 1e-12, mu 1, direct
    convolution, no diagonal acceleration.  fix[] is in model order (eta0, B,
    vlos, dopp, aa, gm, az, S0, S1, mac, alfa) although the file lists S0, S1
    first."""
    with open(path) as f:
        lines = f.read().splitlines()
    if len(lines) < 42:
        raise ValueError(f"{path}: a control file has 42 lines, found {len(lines)}")
    v = [_field(l) for l in lines]

    def as_int(s, default=0):
        try:
            return int(s.split()[0])
        except (ValueError, IndexError):
            return default

    def as_float(s, default):
        try:
            return float(s.split()[0])
        except (ValueError, IndexError):
            return default

    cfg = {"cycles": as_int(v[0]), "observed": v[1], "stray_light": v[2], "psf": v[3], "wavelength": v[4],
           "atomic": v[5], "guess": v[7]}
    cfg["weights"] = [as_float(v[9 + k], 1.0) for k in range(4)]
    fix = [0] * 11
    order = (7, 8, 0, 1, 2, 5, 6, 3, 4, 9)  # lines 15-24
    for k, idx in enumerate(order):
        fix[idx] = as_int(v[14 + k])
    fix[10] = as_int(v[35])
    cfg["fix"] = fix
    cfg["mu"] = as_float(v[36], 1.0)
    sn = as_int(v[37])
    cfg["sn"] = sn
    cfg["noise"] = (1.0 / sn) ** 2 if sn != 0 else 0.001 ** 2
    cfg["ilambda"] = as_float(v[39], 0.1)
    cfg["use_fft"] = as_int(v[40])
    cfg["logclambda"] = as_int(v[41])
    cfg["toplim"] = 1e-12
    # PSF: a file, a numeric FWHM in mA, or nothing (readConfig.c:474-512)
    psf = cfg["psf"]
    base = os.path.dirname(os.path.abspath(path))
    if psf and os.path.exists(os.path.join(base, psf)):
        cfg["psf_file"] = os.path.join(base, psf)
        cfg["psf_fwhm"] = None
    else:
        try:
            fw = float(psf) if psf else 0.0
        except ValueError:
            fw = 0.0
        cfg["psf_file"] = None
        cfg["psf_fwhm"] = fw if fw != 0 and not math.isnan(fw) else None
    return cfg


def cube_fits_bytes(data: np.ndarray, ctypes_: list | None = None) -> bytes:
    """A spectro cube as a FITS file (primary HDU, BITPIX = -32, big-endian):
    ``data`` is a float32 array of numpy shape (NAXIS4, NAXIS3, NAXIS2, NAXIS1);
    ``ctypes_`` gives CTYPE1..4 ('WAVE-GRI', 'STOKES', 'HPLN-TAN', 'HPLT-TAN' in
    the reference's default order), or None for a header without them."""
    dims = list(data.shape[::-1])
    cards = ["SIMPLE  =                    T", "BITPIX  =                  -32", f"NAXIS   = {len(dims):20d}"]
    cards += [f"NAXIS{i + 1}  = {d:20d}" for i, d in enumerate(dims)]
    if ctypes_:
        cards += [f"CTYPE{i + 1}  = '{c:<8s}'" for i, c in enumerate(ctypes_)]
    cards.append("END")
    hdr = "".join(c.ljust(80) for c in cards).encode("ascii")
    hdr += b" " * (-len(hdr) % 2880)
    body = np.ascontiguousarray(data, dtype=">f4").tobytes()
    body += b"\0" * (-len(body) % 2880)
    return hdr + body


# ---- small FITS arrays (stray light, wavelengths) ----
def fits_array(raw) -> tuple[list, dict, np.ndarray]:
    """(naxes, cards, data) of a primary-HDU FITS image of BITPIX -32 or -64:
    naxes in FITS order (NAXIS1 fastest), data as a float64 numpy array of shape
    naxes[::-1]."""
    raw = bytes(raw)
    cards, pos = {}, 0
    while True:
        if pos + 2880 > len(raw):
            raise ValueError("FITS header without END")
        block = raw[pos:pos + 2880]
        pos += 2880
        done = False
        for i in range(36):
            card = block[80 * i:80 * (i + 1)].decode("ascii", "replace")
            key = card[:8].strip()
            if key == "END":
                done = True
                break
            if card[8:10] == "= ":
                val = card[10:].split("/")[0].strip()
                cards[key] = val.strip("'").strip() if val.startswith("'") else val
        if done:
            break
    bitpix = int(cards["BITPIX"])
    if bitpix not in (-32, -64):
        raise ValueError(f"BITPIX {bitpix}: float images only")
    naxes = [int(cards[f"NAXIS{i + 1}"]) for i in range(int(cards["NAXIS"]))]
    n = int(np.prod(naxes))
    dt = ">f4" if bitpix == -32 else ">f8"
    data = np.frombuffer(raw, dtype=dt, count=n, offset=pos).astype(np.float64)
    return naxes, cards, data.reshape(naxes[::-1])


def read_stray_light_fits(source):
    """A stray-light FITS file as readFitsStrayLightFile reads it: a 2-D array
    (nlambda x 4 in either axis order; the longer axis is wavelength) gives one
    profile [4][nlambda] (float32) for every pixel; a 4-D cube gives a profile
    per pixel, [npix][4][nlambda] in the cube ingest's pixel order (a CUDA
    tensor, reordered on the device like an observed cube), for
    PM_SLIGHT_PER_PIXEL (pmilos.c:1293)."""
    raw = open(source, "rb").read() if isinstance(source, (str, os.PathLike)) else bytes(source)
    naxes, _, data = fits_array(raw)
    if len(naxes) == 2:
        if naxes[0] >= naxes[1]:  # NAXIS1 = wavelength: stored [stokes][lambda]
            return np.ascontiguousarray(data, dtype=np.float32)
        return np.ascontiguousarray(data.T, dtype=np.float32)  # NAXIS1 = Stokes
    if len(naxes) == 4:
        from . import ingest_fits

        return ingest_fits(raw)
    raise ValueError(f"a stray-light file has 2 or 4 axes, not {len(naxes)}")


def read_wavelength_fits(source):
    """A wavelength FITS file.  2-D (NAXIS1 = nlambda, NAXIS2 = 2): the first row
    holds the line's index in the atomic parameter file, the second the
    wavelengths [A] -- readFitsLambdaToArray's reading; returns (index, lambda
    [nlambda]).  4-D: one grid per pixel for pm_invert_batch_grids.  The
    reference documents this form (README, "Wavelength grid file (.fits)") but
    its reader does not load it; read here with the axis order of that reader's
    comment, NAXIS1 = rows, NAXIS2 = columns, NAXIS3 = wavelength, NAXIS4 = 1
    (or by CTYPE HPLN-TAN / HPLT-TAN / WAVE-GRI when present); returns (None,
    lambda [npix][nlambda]), pixel = column * rows + row as in the cube ingest."""
    raw = open(source, "rb").read() if isinstance(source, (str, os.PathLike)) else bytes(source)
    naxes, cards, data = fits_array(raw)
    if len(naxes) == 2:
        flat = data.reshape(-1)
        nl = naxes[0]
        return int(flat[nl - 1]), flat[nl:2 * nl].copy()
    if len(naxes) != 4:
        raise ValueError(f"a wavelength file has 2 or 4 axes, not {len(naxes)}")
    role = {"HPLN-TAN": "row", "HPLT-TAN": "col", "WAVE-GRI": "lam"}
    axes = {}
    for i in range(4):
        r = role.get(cards.get(f"CTYPE{i + 1}", ""))
        if r:
            axes[r] = i
    if len(axes) != 3:
        axes = {"row": 0, "col": 1, "lam": 2}
    rest = [i for i in range(4) if i not in axes.values()]
    if naxes[rest[0]] != 1:
        raise ValueError("the fourth axis of a per-pixel wavelength file has one element")
    # numpy axis of FITS axis a is 3 - a; target order (col, row, lambda)
    t = np.transpose(data, (3 - axes["col"], 3 - axes["row"], 3 - axes["lam"], 3 - rest[0]))
    return None, np.ascontiguousarray(t.reshape(naxes[axes["col"]] * naxes[axes["row"]], naxes[axes["lam"]]))
