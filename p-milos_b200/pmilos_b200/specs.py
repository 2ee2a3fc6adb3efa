"""Benchmark workload definitions in plain numpy (no library calls).

The shapes and value distributions of the five benchmark configurations: the
line (Fe I 6173.3354 A or 6302.4936 A, 5P1.0-5D0.0, a normal Zeeman triplet
with g_eff = 2.5), the wavelength grid (.grid-file rules of milos.c:176-196),
the instrumental PSF table (a zero-mean, unit-area Gaussian sampled at 1 mA like
run/CRISP_6173_1mA.psf), the seeded per-pixel atmospheres and the fixed initial
guess.  The reference's CRISP example cubes are not distributed with it, so
seeded synthetic cubes with these distributions stand in for them.

This module imports nothing from the package, so a process that must not load
the CUDA library (the benchmark's reference arm) can load it by file path.
"""
from __future__ import annotations

import numpy as np

FE6173 = 6173.3354
FE6302 = 6302.4936
TRIPLET = (2.0, 1.0, 1.0, 2.0, 2.0, 0.0)  # 5P1.0 - 5D0.0 after readFileCuanticLines' decoding
GUESS = np.array([8.0, 400.0, 0.0, 0.03, 0.1, 30.0, 30.0, 0.25, 0.75, 0.0, 1.0])
QUIET_SUN_B0 = np.array([13.0, 0.0, 0.2, 0.035, 0.19, 30.0, 30.0, 0.26, 0.74, 0.0, 1.0])
NOISE_SIGMA = 1e-3
SN = 1000
DEFAULT_NPIX = {0: 64 * 64, 1: 256 * 256, 2: 1024 * 1024, 3: 256 * 256, 4: 4096 * 4096}


def grid_spec(cfg: int, which: int = 2):
    """(initial mA, step mA, final mA, lambda0 A) of configuration ``cfg``'s grid;
    configuration 3 has three grids (6, 15 and 30 points), ``which`` picks one."""
    if cfg == 4:
        return -1204.0, 21.5, 1182.5, FE6302
    if cfg == 3:
        return [(-172.5, 69.0, 172.5), (-350.0, 50.0, 350.0), (-350.0, 25.0, 375.0)][which] + (FE6173,)
    return -350.0, 25.0, 375.0, FE6173


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


def gaussian_psf_table(fwhm_ma: float, half_range_ma: float = 1500.0, step_ma: float = 1.0):
    """A zero-mean, unit-area Gaussian sampled like run/CRISP_6173_1mA.psf."""
    x = np.arange(-half_range_ma, half_range_ma + step_ma / 2, step_ma)
    sig = fwhm_ma / (2.0 * np.sqrt(2.0 * np.log(2.0)))
    y = np.exp(-0.5 * (x / sig) ** 2)
    y /= y.sum() * step_ma
    return x, y


def psf_route(cfg: int):
    """How configuration ``cfg`` builds its PSF: None (no PSF), ("table", fwhm)
    for the 1 mA .psf-file route, or ("fwhm", fwhm) for the numeric-FWHM route
    (configuration 3: its 6-point grid has no zero sample)."""
    return {1: ("table", 60.0), 2: ("table", 60.0), 3: ("fwhm", 60.0), 4: ("table", 25.0)}.get(cfg)


def nterms_fix_guess(cfg: int):
    """(NTERMS, fix[11], initial guess) of configuration ``cfg``: 9 free
    parameters, or 10 with the filling factor (configuration 2)."""
    guess = GUESS.copy()
    if cfg == 2:
        guess[10] = 0.9
        return 10, [1] * 9 + [0, 1], guess
    return 9, [1] * 9 + [0, 0], guess


def truth_models(cfg: int, npix: int, rng: np.random.Generator) -> np.ndarray:
    """Seeded per-pixel atmospheres [npix][11] of configuration ``cfg``."""
    n = npix
    m = np.zeros((n, 11))
    m[:, 0] = rng.uniform(1, 20, n)
    m[:, 1] = rng.uniform(0, 3000, n)
    m[:, 2] = rng.uniform(-3, 3, n)
    m[:, 3] = rng.uniform(0.02, 0.05, n)
    m[:, 4] = rng.uniform(0.01, 0.5, n)
    m[:, 5] = rng.uniform(0, 180, n)
    m[:, 6] = rng.uniform(0, 180, n)
    m[:, 7] = rng.uniform(0.1, 0.4, n)
    m[:, 8] = rng.uniform(0.4, 0.9, n)
    m[:, 9] = 0.0
    m[:, 10] = 1.0
    if cfg in (2, 3):
        weak = rng.uniform(0, 1, n) < 0.7
        m[weak, 1] = rng.uniform(0, 200, int(weak.sum()))
        m[weak, 0] = rng.uniform(1, 5, int(weak.sum()))
        m[~weak, 1] = rng.uniform(1500, 3500, int((~weak).sum()))
    if cfg == 2:
        m[:, 10] = 1.0 - rng.uniform(0, 0.3, n)
    return m
