"""Generate the golden fixtures of tests/golden/ from the REFERENCE itself.

Run in a container where the reference tree exists (its sources are compiled by
oracle/Makefile into oracle/_ref/):

    python tests/golden/make_golden.py --reference <the reference tree>

(or with PM_REFERENCE_SRC set to its src/ directory)

Writes
  kat_synthesis.npz   the reference's own known-answer test (test/synthesis.mtrol:
                      obs.mod + malla.grid + LINES entry 1 + straylight.fits ->
                      synthesis_results.per), inputs and expected profiles
  ref_cases.npz       per configuration (0, 1, 2; 48 pixels each): grid, PSF taps,
                      truth models, observed profiles, and the reference's
                      inversion results in both builds (REAL = float / double),
                      plus mil_sinrf + me_der outputs at 12 models
  ref_psf.npz         the reference's fgauss_WL and interpolationLinearPSF on the
                      configuration grids (host precompute pinning)
  fits_cases.npz      the reference's FITS cube reader (readFitsSpectroImage over
                      a CFITSIO read shim) on small cubes in eight axis orders,
                      with and without CTYPE cards: file bytes and output
  ref_cases_wide.npz  the same per-case content on grids wider than one warp:
                      w112 (112 points of Fe I 6302 at 21.5 mA, 25 mA PSF, the
                      large-cube configuration) and w49 (the known-answer test's
                      49-point grid with a 60 mA PSF, stray light and the filling
                      factor inverted); 16 pixels each
  fits_aux_cases.npz  the reference's stray-light reader (readFitsStrayLightFile)
                      on 2-D profiles in both axis orders and on 4-D cubes, and
                      its wavelength reader (readFitsLambdaToArray) on 2-D files
                      of float64 and float32: file bytes and output
  ref_cases_zeeman.npz  a Zeeman multiplet, Fe I 6301.5012 (5P2.0-5D2.0: five pi
                      and four sigma components per group), 60 mA PSF: z9 and
                      z10 on a 30-point grid, zw9 on 49 points and zw10 on 112
                      points (25 mA steps); the *10 cases add stray light and
                      invert the filling factor; with v_mac inverted: zm10 on
                      30 points and zmw11 on 112 (stray light and filling
                      factor too); 24 pixels and 8 synthesis models each (16
                      and 4 on the wide grids)
  ref_cases_mac.npz   macroturbulence on the 30-point grid: m10 (v_mac inverted,
                      60 mA PSF), m10n (the same without PSF), m11 (v_mac and
                      the filling factor inverted, stray light), mfix (v_mac
                      fixed at 1.2 km/s); 24 pixels and 8 synthesis models each;
                      and on wider grids: mw10 (as m10, 49 points) and mw11 (as
                      m11, 112 points), 16 pixels and 4 models each
The fixtures are what the CPU test-suite compares the oracle restatement and the
host precompute with, so those tests need neither the reference nor a GPU.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "p-milos_b200"))

import pyoracle as po  # noqa: E402
from fitsmini import read_fits_f32  # noqa: E402

TRIPLET = np.array([1.0, 2.0, 1.0, 1.0, 2.0, 2.0, 0.0])
GUESS = np.array([8.0, 400.0, 0.0, 0.03, 0.1, 30.0, 30.0, 0.25, 0.75, 0.0, 1.0])


def grid(ini, step, fin, l0):
    nl = int((fin - ini) / step) + 1
    offs = np.zeros(nl)
    offs[0] = ini
    for i in range(1, nl):
        offs[i] = offs[i - 1] + step
    lam = np.zeros(nl)
    lam[0] = l0 + ini / 1000.0
    for i in range(1, nl):
        lam[i] = lam[i - 1] + step / 1000.0
    return offs, lam


def gauss_table(fwhm, half=1500.0, step=1.0):
    x = np.arange(-half, half + step / 2, step)
    sig = fwhm / (2.0 * np.sqrt(2.0 * np.log(2.0)))
    y = np.exp(-0.5 * (x / sig) ** 2)
    y /= y.sum() * step
    return x, y


def kat(refdir):
    t = os.path.join(refdir, "test")
    gold = np.loadtxt(os.path.join(t, "synthesis_results.per"))
    _, dims, sl = read_fits_f32(os.path.join(t, "straylight.fits"))
    offs, lam = grid(-600.0, 25.0, 600.0, 6173.3356)
    model = np.array([14.0, 1200.0, 0.5, 0.07, 0.05, 130.0, 25.0, 0.2, 0.75, 0.0, 0.85])
    return dict(lam=lam, offs=offs, lambda0=6173.3356, cuantic=TRIPLET, model=model, slight=sl.reshape(4, -1),
                expected=gold[:, 2:].T.copy(), expected_offsets=gold[:, 1].copy(), nterms=10)


# grid (ini, step, fin, lambda0), PSF FWHM [mA] (None = no PSF), stray light + filling factor
CASE_SPECS = {
    0: ((-350.0, 25.0, 375.0, 6173.3354), None, False),
    1: ((-350.0, 25.0, 375.0, 6173.3354), 60.0, False),
    2: ((-350.0, 25.0, 375.0, 6173.3354), 60.0, True),
    112: ((-1204.0, 21.5, 1182.5, 6302.4936), 25.0, False),
    49: ((-600.0, 25.0, 600.0, 6173.3356), 60.0, True),
}


# name: PSF FWHM [mA] or None, stray light + filling factor, v_mac inverted
MAC_SPECS = {
    "m10": (60.0, False, True),
    "m10n": (None, False, True),
    "m11": (60.0, True, True),
    "mfix": (60.0, False, False),
    "mw10": (60.0, False, True),
    "mw11": (60.0, True, True),
}
# grids of the cases that are not on the configuration-1 grid (25 mA steps)
MAC_GRIDS = {"mw10": (-600.0, 25.0, 600.0), "mw11": (-1387.5, 25.0, 1387.5)}


def mac_case(name, npix=24, nsynth=8):
    """Macroturbulence on the configuration-1 grid (49 and 112 points for the mw
    cases): truths with v_mac in U(0.3, 3) km/s, guess v_mac = 1 (1.2 and fixed
    for mfix)."""
    fwhm, stray, free = MAC_SPECS[name]
    rng = np.random.default_rng(sum(ord(ch) for ch in name) + 2000)
    (ini, step, fin, l0) = CASE_SPECS[1][0]
    if name in MAC_GRIDS:
        ini, step, fin = MAC_GRIDS[name]
    offs, lam = grid(ini, step, fin, l0)
    psf = None
    if fwhm is not None:
        x, y = gauss_table(fwhm)
        psf = po.Reference(po.LineSetup(lam, l0, TRIPLET, None, 9), "f64").interp_psf(x, y, offs, 0.0)
    K = 11 if stray else 10
    fix = [1] * 9 + [1 if free else 0, 1 if stray else 0]
    guess = GUESS.copy()
    guess[9] = 1.0 if free else 1.2
    if stray:
        guess[10] = 0.9
    truth = np.zeros((npix, 11))
    truth[:, 0] = rng.uniform(1, 20, npix)
    truth[:, 1] = rng.uniform(0, 3000, npix)
    truth[:, 2] = rng.uniform(-3, 3, npix)
    truth[:, 3] = rng.uniform(0.02, 0.05, npix)
    truth[:, 4] = rng.uniform(0.01, 0.5, npix)
    truth[:, 5] = rng.uniform(0, 180, npix)
    truth[:, 6] = rng.uniform(0, 180, npix)
    truth[:, 7] = rng.uniform(0.1, 0.4, npix)
    truth[:, 8] = rng.uniform(0.4, 0.9, npix)
    truth[:, 9] = rng.uniform(0.3, 3.0, npix) if free else 1.2
    truth[:, 10] = 1.0 - rng.uniform(0, 0.3, npix) if stray else 1.0
    slight = None
    if stray:
        r9 = po.Reference(po.LineSetup(lam, l0, TRIPLET, psf, 9), "f64")
        slight, _ = r9.synth(np.array([13.0, 0.0, 0.2, 0.035, 0.19, 30.0, 30.0, 0.26, 0.74, 0.0, 1.0]), rf=False)
        slight = slight.astype(np.float32).astype(np.float64)
    setup = po.LineSetup(lam, l0, TRIPLET, psf, K)
    out = dict(lam=lam, offs=offs, lambda0=l0, psf=np.zeros(0) if psf is None else psf, truth=truth, guess=guess,
               fix=np.array(fix, dtype=np.int32), nterms=K, slight=np.zeros(0) if slight is None else slight)
    ref64 = po.Reference(setup, "f64")
    obs = np.array([ref64.synth(m, slight, fix=fix, rf=False)[0] for m in truth], dtype=np.float32)
    obs += rng.normal(0, 1e-3, obs.shape).astype(np.float32)
    out["obs"] = obs
    for flav in ("f32", "f64"):
        ref = po.Reference(setup, flav)
        noise = float(np.float32(np.float32(1.0 / 1000) ** 2)) if flav == "f32" else (1.0 / 1000) ** 2
        r = ref.invert(obs, guess, slight=slight, fix=fix, noise=noise)
        for k in ("models", "chisq", "iters", "spectra"):
            out[f"{flav}_{k}"] = r[k]
        models = truth[:nsynth].copy()
        sp, rf = zip(*[ref.synth(m, slight, fix=fix) for m in models])
        out[f"{flav}_synth_models"] = models
        out[f"{flav}_synth"] = np.array(sp)
        out[f"{flav}_rf"] = np.array(rf)
    return out


MULTIPLET = np.array([1.0, 2.0, 1.0, 2.0, 2.0, 2.0, 2.0])  # 5P 2.0 - 5D 2.0
LAMBDA_6301 = 6301.5012
G30, G49, G112 = (-350.0, 25.0, 375.0), (-600.0, 25.0, 600.0), (-1387.5, 25.0, 1387.5)
# name: grid, stray light + filling factor, v_mac inverted
ZEEMAN_SPECS = {"z9": (G30, False, False), "z10": (G30, True, False), "zw9": (G49, False, False),
                "zw10": (G112, True, False), "zm10": (G30, False, True), "zmw11": (G112, True, True)}


def zeeman_case(name, npix=24, nsynth=8):
    """A multiplet line (LINES entry 2 of the reference's run directory) with the
    configuration-1 atmospheres; stray light and the filling factor, and v_mac
    in U(0.3, 3) km/s inverted from a guess of 1, as ZEEMAN_SPECS says."""
    grid_spec, stray, mac = ZEEMAN_SPECS[name]
    rng = np.random.default_rng(sum(ord(ch) for ch in name) + 3000)
    offs, lam = grid(*grid_spec, LAMBDA_6301)
    x, y = gauss_table(60.0)
    psf = po.Reference(po.LineSetup(lam, LAMBDA_6301, MULTIPLET, None, 9), "f64").interp_psf(x, y, offs, 0.0)
    K = 9 + int(stray) + int(mac)
    fix = [1] * 9 + [1 if mac else 0, 1 if stray else 0]
    guess = GUESS.copy()
    if mac:
        guess[9] = 1.0
    if stray:
        guess[10] = 0.9
    truth = np.zeros((npix, 11))
    truth[:, 0] = rng.uniform(1, 20, npix)
    truth[:, 1] = rng.uniform(0, 3000, npix)
    truth[:, 2] = rng.uniform(-3, 3, npix)
    truth[:, 3] = rng.uniform(0.02, 0.05, npix)
    truth[:, 4] = rng.uniform(0.01, 0.5, npix)
    truth[:, 5] = rng.uniform(0, 180, npix)
    truth[:, 6] = rng.uniform(0, 180, npix)
    truth[:, 7] = rng.uniform(0.1, 0.4, npix)
    truth[:, 8] = rng.uniform(0.4, 0.9, npix)
    if mac:
        truth[:, 9] = rng.uniform(0.3, 3.0, npix)
    truth[:, 10] = 1.0 - rng.uniform(0, 0.3, npix) if stray else 1.0
    slight = None
    if stray:
        r9 = po.Reference(po.LineSetup(lam, LAMBDA_6301, MULTIPLET, psf, 9), "f64")
        slight, _ = r9.synth(np.array([13.0, 0.0, 0.2, 0.035, 0.19, 30.0, 30.0, 0.26, 0.74, 0.0, 1.0]), rf=False)
        slight = slight.astype(np.float32).astype(np.float64)
    setup = po.LineSetup(lam, LAMBDA_6301, MULTIPLET, psf, K)
    out = dict(lam=lam, offs=offs, lambda0=LAMBDA_6301, cuantic=MULTIPLET, psf=psf, truth=truth, guess=guess,
               fix=np.array(fix, dtype=np.int32), nterms=K, slight=np.zeros(0) if slight is None else slight)
    ref64 = po.Reference(setup, "f64")
    out["cuantic_pattern"] = ref64.cuantic()
    obs = np.array([ref64.synth(m, slight, fix=fix, rf=False)[0] for m in truth], dtype=np.float32)
    obs += rng.normal(0, 1e-3, obs.shape).astype(np.float32)
    out["obs"] = obs
    for flav in ("f32", "f64"):
        ref = po.Reference(setup, flav)
        noise = float(np.float32(np.float32(1.0 / 1000) ** 2)) if flav == "f32" else (1.0 / 1000) ** 2
        r = ref.invert(obs, guess, slight=slight, fix=fix, noise=noise)
        for k in ("models", "chisq", "iters", "spectra"):
            out[f"{flav}_{k}"] = r[k]
        models = truth[:nsynth].copy()
        sp, rf = zip(*[ref.synth(m, slight, fix=fix) for m in models])
        out[f"{flav}_synth_models"] = models
        out[f"{flav}_synth"] = np.array(sp)
        out[f"{flav}_rf"] = np.array(rf)
    return out


def case(cfg, seed, npix=48, nsynth=12):
    rng = np.random.default_rng(1000 + cfg)
    (ini, step, fin, l0), fwhm, stray = CASE_SPECS[cfg]
    offs, lam = grid(ini, step, fin, l0)
    psf = None
    setup0 = po.LineSetup(lam, l0, TRIPLET, None, 9)
    if fwhm is not None:
        x, y = gauss_table(fwhm)
        psf = po.Reference(setup0, "f64").interp_psf(x, y, offs, 0.0)
    K = 10 if stray else 9
    fix = [1] * 9 + [0, 1 if K == 10 else 0]
    guess = GUESS.copy()
    if K == 10:
        guess[10] = 0.9
    truth = np.zeros((npix, 11))
    truth[:, 0] = rng.uniform(1, 20, npix)
    truth[:, 1] = rng.uniform(0, 3000, npix)
    truth[:, 2] = rng.uniform(-3, 3, npix)
    truth[:, 3] = rng.uniform(0.02, 0.05, npix)
    truth[:, 4] = rng.uniform(0.01, 0.5, npix)
    truth[:, 5] = rng.uniform(0, 180, npix)
    truth[:, 6] = rng.uniform(0, 180, npix)
    truth[:, 7] = rng.uniform(0.1, 0.4, npix)
    truth[:, 8] = rng.uniform(0.4, 0.9, npix)
    truth[:, 10] = 1.0
    slight = None
    if stray:
        weak = np.arange(npix) % 10 < 7
        truth[weak, 1] = rng.uniform(0, 200, weak.sum())
        truth[weak, 0] = rng.uniform(1, 5, weak.sum())
        truth[~weak, 1] = rng.uniform(1500, 3500, (~weak).sum())
        truth[:, 10] = 1.0 - rng.uniform(0, 0.3, npix)
        r9 = po.Reference(po.LineSetup(lam, l0, TRIPLET, psf, 9), "f64")
        slight, _ = r9.synth(np.array([13.0, 0.0, 0.2, 0.035, 0.19, 30.0, 30.0, 0.26, 0.74, 0.0, 1.0]), rf=False)
        slight = slight.astype(np.float32).astype(np.float64)
    setup = po.LineSetup(lam, l0, TRIPLET, psf, K)
    out = dict(lam=lam, offs=offs, lambda0=l0, psf=np.zeros(0) if psf is None else psf, truth=truth, guess=guess,
               fix=np.array(fix, dtype=np.int32), nterms=K, slight=np.zeros(0) if slight is None else slight)
    ref64 = po.Reference(setup, "f64")
    obs = np.array([ref64.synth(m, slight, fix=fix, rf=False)[0] for m in truth], dtype=np.float32)
    obs += rng.normal(0, 1e-3, obs.shape).astype(np.float32)
    if cfg == 0:  # ghost points: two masked wavelengths in two pixels
        obs[3, :, 0] = -2.0
        obs[5, 3, 7] = -1.5
    out["obs"] = obs
    for flav in ("f32", "f64"):
        ref = po.Reference(setup, flav)
        noise = float(np.float32(np.float32(1.0 / 1000) ** 2)) if flav == "f32" else (1.0 / 1000) ** 2
        r = ref.invert(obs, guess, slight=slight, fix=fix, noise=noise)
        for k in ("models", "chisq", "iters", "spectra"):
            out[f"{flav}_{k}"] = r[k]
        models = truth[:nsynth].copy()
        sp, rf = zip(*[ref.synth(m, slight, fix=fix) for m in models])
        out[f"{flav}_synth_models"] = models
        out[f"{flav}_synth"] = np.array(sp)
        out[f"{flav}_rf"] = np.array(rf)
    return out


# FITS cubes in several axis orders, with and without CTYPE cards: (order of
# roles for FITS axes 1..4, CTYPEs written?).  R = rows, C = cols, L = wavelength,
# S = Stokes.
FITS_ORDERS = [("LSRC", True), ("SLRC", True), ("RCLS", True), ("CRSL", True), ("LRSC", True),
               ("LSRC", False), ("RCLS", False), ("SRLC", False)]
CTYPE_OF = {"R": "HPLN-TAN", "C": "HPLT-TAN", "L": "WAVE-GRI", "S": "STOKES"}


def fits_cases(tmpdir):
    """The reference's reader on small synthetic cubes: the file bytes and its
    output (pmilos' forParallel layout) per axis order."""
    rng = np.random.default_rng(77)
    size = {"R": 9, "C": 11, "L": 7, "S": 4}
    out = {}
    for k, (order, with_ctype) in enumerate(FITS_ORDERS):
        dims = [size[r] for r in order]
        data = rng.normal(size=dims[::-1]).astype(np.float32)
        ct = [CTYPE_OF[r] for r in order] if with_ctype else None
        raw = po.fits_bytes(data, ct)
        path = os.path.join(tmpdir, f"cube{k}.fits")
        open(path, "wb").write(raw)
        cube, rows, cols = po.reference_fits_read(path, size["L"], size["R"] * size["C"])
        out[f"f{k}_bytes"] = np.frombuffer(raw, dtype=np.uint8)
        out[f"f{k}_ref"] = cube
        out[f"f{k}_order"] = np.array(order)
        out[f"f{k}_ctype"] = np.array(with_ctype)
        out[f"f{k}_rows_cols"] = np.array([rows, cols])
    return out


def fits_image_bytes(data: np.ndarray, bitpix: int = -32, ctypes_: list | None = None) -> bytes:
    """A primary-HDU FITS image of numpy shape (NAXISn, ..., NAXIS1)."""
    dims = list(data.shape[::-1])
    cards = ["SIMPLE  =                    T", f"BITPIX  = {bitpix:20d}", f"NAXIS   = {len(dims):20d}"]
    cards += [f"NAXIS{i + 1}  = {d:20d}" for i, d in enumerate(dims)]
    if ctypes_:
        cards += [f"CTYPE{i + 1}  = '{c:<8s}'" for i, c in enumerate(ctypes_)]
    cards.append("END")
    hdr = "".join(c.ljust(80) for c in cards).encode("ascii")
    hdr += b" " * (-len(hdr) % 2880)
    body = np.ascontiguousarray(data, dtype=">f4" if bitpix == -32 else ">f8").tobytes()
    body += b"\0" * (-len(body) % 2880)
    return hdr + body


def fits_aux_cases(tmpdir):
    """The reference's stray-light and wavelength readers on small files."""
    rng = np.random.default_rng(78)
    out = {}
    # stray light, 2-D: (Stokes, lambda) or (lambda, Stokes) in numpy order
    for k, shape in enumerate([(4, 30), (30, 4), (4, 7), (15, 4)]):
        data = rng.normal(size=shape).astype(np.float32)
        raw = fits_image_bytes(data)
        path = os.path.join(tmpdir, f"sl2d{k}.fits")
        open(path, "wb").write(raw)
        arr, nl, ns, nx, ny = po.reference_fits_straylight(path)
        out[f"s2_{k}_bytes"] = np.frombuffer(raw, dtype=np.uint8)
        out[f"s2_{k}_ref"] = arr.reshape(ns, nl)
    # stray light, 4-D cubes (the RCLS order takes the reference's special branch)
    size = {"R": 5, "C": 6, "L": 7, "S": 4}
    for k, (order, ct) in enumerate([("LSRC", True), ("SLRC", True), ("CRSL", True), ("LSRC", False)]):
        dims = [size[r] for r in order]
        data = rng.normal(size=dims[::-1]).astype(np.float32)
        raw = fits_image_bytes(data, -32, [CTYPE_OF[r] for r in order] if ct else None)
        path = os.path.join(tmpdir, f"sl4d{k}.fits")
        open(path, "wb").write(raw)
        arr, nl, ns, nx, ny = po.reference_fits_straylight(path)
        out[f"s4_{k}_bytes"] = np.frombuffer(raw, dtype=np.uint8)
        out[f"s4_{k}_ref"] = arr.reshape(nx * ny, ns, nl)
        out[f"s4_{k}_order"] = np.array(order)
    # wavelength files, 2-D: row 1 the line index, row 2 the wavelengths
    offs, lam = grid(-350.0, 25.0, 375.0, 6173.3354)
    for k, bitpix in enumerate((-64, -32)):
        data = np.stack([np.full(lam.size, 1.0), lam])
        raw = fits_image_bytes(data, bitpix)
        path = os.path.join(tmpdir, f"lam{k}.fits")
        open(path, "wb").write(raw)
        idx, v = po.reference_fits_lambda(path)
        out[f"l2_{k}_bytes"] = np.frombuffer(raw, dtype=np.uint8)
        out[f"l2_{k}_index"] = np.array(idx)
        out[f"l2_{k}_ref"] = v
    return out


def psf_pins():
    ref = po.Reference(po.LineSetup(*grid(-350.0, 25.0, 375.0, 6173.3354)[1:], 6173.3354, TRIPLET, None, 9), "f64")
    out = {}
    for name, (ini, step, fin, l0), fw in (("c1", (-350.0, 25.0, 375.0, 6173.3354), 60.0),
                                          ("c3a", (-172.5, 69.0, 172.5, 6173.3354), 60.0),
                                          ("c3b", (-350.0, 50.0, 350.0, 6173.3354), 60.0),
                                          ("c4", (-1204.0, 21.5, 1182.5, 6302.4936), 25.0),
                                          ("kat", (-600.0, 25.0, 600.0, 6173.3356), 60.0)):
        offs, lam = grid(ini, step, fin, l0)
        n = lam.size
        out[f"{name}_lam"] = lam
        out[f"{name}_offs"] = offs
        out[f"{name}_fgauss"] = ref.fgauss_wl(fw, lam[1] - lam[0], lam[0], lam[n // 2], n)
        x, y = gauss_table(fw)
        # the milos.c:332-340 re-centring: offset when the zero sample is not nl/2
        posWL = 0
        for i in range(n):
            if posWL:
                break
            if abs(np.trunc(offs[i])) == 0:
                posWL = i
        offset = 0.0 if posWL == n // 2 else ((n // 2 - posWL) * (step / 1000.0)) * 1000
        out[f"{name}_table_x"] = x
        out[f"{name}_table_y"] = y
        out[f"{name}_interp"] = ref.interp_psf(x, y, offs, offset)
        out[f"{name}_fwhm"] = fw
    return out


def lines_cases(reference):
    """create_cuantic (create_cuantic.c:60-294) of every entry of the reference's
    run/LINES file: the entry's text and the reference's pattern (N_PI, N_SIG,
    GL, GU, GEFF, FO, NUB, NUP, NUR, WEB, WEP, WER)."""
    from pmilos_b200.files import parse_lines_entry
    out = {}
    with open(os.path.join(reference, "run", "LINES")) as f:
        entries = [ln.rstrip("\n") for ln in f if ln.strip()]
    for text in entries:
        # entry 5's "7k" reads as K: L = 7 (readFileCuanticLines leaves L unset for it)
        idx, lam0, q = parse_lines_entry(text)
        lam = lam0 + np.linspace(-0.35, 0.35, 30)
        ref = po.Reference(po.LineSetup(lam, lam0, np.array([1.0, *q]), None, 9), "f64")
        out[f"l{idx}_text"] = np.array(text)
        out[f"l{idx}_lambda0"] = lam0
        out[f"l{idx}_quantum"] = np.array(q, dtype=np.float64)
        out[f"l{idx}_pattern"] = ref.cuantic()
    return out


def classical_only_cases():
    """The classical-estimates-only mode (NumberOfCycles < 0, milos.c:486-501:
    estimacionesClasicas with forInitialUse = 0 from the initial model) on the
    observed cubes of ref_cases.npz (configurations 0, 1, 2) and
    ref_cases_wide.npz (49 and 112 points), both precisions."""
    out = {}
    for fname, names in (("ref_cases.npz", ("c0", "c1", "c2")), ("ref_cases_wide.npz", ("w49", "w112"))):
        src = np.load(os.path.join(HERE, fname))
        for name in names:
            g = lambda k: src[f"{name}_{k}"]
            lam, obs, guess = g("lam"), g("obs"), g("guess")
            l0 = float(g("lambda0")) if f"{name}_lambda0" in src.files else CASE_SPECS[int(name[1])][0][3]
            cu = TRIPLET
            for flav in ("f32", "f64"):
                ref = po.Reference(po.LineSetup(lam, l0, cu, None, 9), flav)
                out[f"{name}_{flav}_models"] = np.array([ref.classical(o, guess, initial_use=False) for o in obs])
            out[f"{name}_lam"], out[f"{name}_lambda0"], out[f"{name}_guess"] = lam, l0, guess
            out[f"{name}_obs"] = obs
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="the reference tree (default: the parent of $PM_REFERENCE_SRC)")
    ap.add_argument("--only", choices=("all", "wide", "mac", "fits", "zeeman", "classical", "lines"), default="all")
    a = ap.parse_args()
    if a.reference is None:
        src = os.environ.get("PM_REFERENCE_SRC")
        if not src:
            ap.error("give --reference <the reference tree> or set PM_REFERENCE_SRC to its src/ directory")
        a.reference = os.path.dirname(os.path.abspath(src))
    os.environ["PM_REFERENCE_SRC"] = os.path.join(a.reference, "src")
    po.build()
    if a.only in ("all", "lines"):
        np.savez_compressed(os.path.join(HERE, "ref_lines.npz"), **lines_cases(a.reference))
        print("ref_lines.npz", os.path.getsize(os.path.join(HERE, "ref_lines.npz")), "bytes")
        if a.only == "lines":
            return
    if a.only in ("all", "classical"):
        np.savez_compressed(os.path.join(HERE, "ref_classical_only.npz"), **classical_only_cases())
        print("ref_classical_only.npz", os.path.getsize(os.path.join(HERE, "ref_classical_only.npz")), "bytes")
        if a.only == "classical":
            return
    import tempfile

    with tempfile.TemporaryDirectory() as td:
        np.savez_compressed(os.path.join(HERE, "fits_aux_cases.npz"), **fits_aux_cases(td))
    print("fits_aux_cases.npz", os.path.getsize(os.path.join(HERE, "fits_aux_cases.npz")), "bytes")
    if a.only == "fits":
        return
    zee = {}
    for name in ZEEMAN_SPECS:
        for k, v in zeeman_case(name, *((24, 8) if ZEEMAN_SPECS[name][0] == G30 else (16, 4))).items():
            zee[f"{name}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "ref_cases_zeeman.npz"), **zee)
    print("ref_cases_zeeman.npz", os.path.getsize(os.path.join(HERE, "ref_cases_zeeman.npz")), "bytes")
    if a.only == "zeeman":
        return
    mac = {}
    for name in MAC_SPECS:
        for k, v in mac_case(name, *((16, 4) if name in MAC_GRIDS else (24, 8))).items():
            mac[f"{name}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "ref_cases_mac.npz"), **mac)
    print("ref_cases_mac.npz", os.path.getsize(os.path.join(HERE, "ref_cases_mac.npz")), "bytes")
    if a.only == "mac":
        return
    files = ["ref_cases_wide.npz"]
    if a.only == "all":
        np.savez_compressed(os.path.join(HERE, "kat_synthesis.npz"), **kat(a.reference))
        cases = {}
        for cfg in (0, 1, 2):
            for k, v in case(cfg, cfg).items():
                cases[f"c{cfg}_{k}"] = v
        np.savez_compressed(os.path.join(HERE, "ref_cases.npz"), **cases)
        np.savez_compressed(os.path.join(HERE, "ref_psf.npz"), **psf_pins())
        files += ["kat_synthesis.npz", "ref_cases.npz", "ref_psf.npz"]
    import tempfile

    with tempfile.TemporaryDirectory() as td:
        np.savez_compressed(os.path.join(HERE, "fits_cases.npz"), **fits_cases(td))
    files.append("fits_cases.npz")
    wide = {}
    for cfg in (112, 49):
        for k, v in case(cfg, cfg, npix=16, nsynth=4).items():
            wide[f"w{cfg}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "ref_cases_wide.npz"), **wide)
    for f in files:
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
