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
"""
from __future__ import annotations

import math
import os
import re

import numpy as np

_LEVELS = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5, "J": 6}
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


def grid_from_malla(initial_ma: float, step_ma: float, final_ma: float, lambda0: float):
    """Wavelength grid as milos.c:176-196 builds it: nl = (final - initial)/step + 1
    (truncated), offsets and wavelengths accumulated sample by sample.
    Returns (offsets [mA], wavelengths [A])."""
    nl = int((final_ma - initial_ma) / step_ma) + 1
    offs = np.zeros(nl)
    offs[0] = initial_ma
    for i in range(1, nl):
        offs[i] = offs[i - 1] + step_ma
    lam = np.zeros(nl)
    lam[0] = lambda0 + initial_ma / 1000.0
    for i in range(1, nl):
        lam[i] = lam[i - 1] + step_ma / 1000.0
    return offs, lam


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
