"""Synthetic workloads with the shapes and value distributions of the benchmark
configurations (the reference's CRISP example cubes are not distributed with it).

Per configuration: a line (Fe I 6173.3354 A or 6302.4936 A, 5P1.0-5D0.0, a normal
Zeeman triplet with g_eff = 2.5), a wavelength grid built like a .grid file, an
instrumental PSF built through the .psf-table route (a Gaussian sampled at
1 mA, as a CRISP-style file) or the numeric-FWHM route, seeded per-pixel
atmospheres, and the fixed initial guess.  Profiles are synthesized on the GPU
with the FP64 form of this library (``synthesize``) and get Gaussian noise of
sigma = 1e-3 in all four Stokes parameters.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import LineData, psf_from_table, psf_gaussian
from .specs import (DEFAULT_NPIX, FE6173, FE6302, GUESS, NOISE_SIGMA, QUIET_SUN_B0, SN, TRIPLET,  # noqa: F401
                    gaussian_psf_table, grid_from_malla, grid_spec, nterms_fix_guess, psf_route)
from .specs import truth_models as _truth_models


@dataclass
class Workload:
    name: str
    cfg: int
    line: LineData
    offs: np.ndarray          # grid offsets [mA]
    lam: np.ndarray           # wavelengths [A]
    psf: np.ndarray | None    # taps on the grid
    npix: int
    seed: int
    nterms: int = 9
    fix: list = field(default_factory=lambda: [1] * 9 + [0, 0])
    guess: np.ndarray = field(default_factory=lambda: GUESS.copy())
    noise: float = (1.0 / SN) ** 2
    miter: int = 50
    slight: np.ndarray | None = None  # [4][nl] stray-light profile (config 2)

    @property
    def nl(self) -> int:
        return int(self.lam.size)


def config(cfg: int, npix: int | None = None, grid: int = 2) -> Workload:
    """Workload spec of benchmark configuration ``cfg`` (0..4)."""
    ini, step, fin, l0 = grid_spec(cfg, grid)
    offs, lam = grid_from_malla(ini, step, fin, l0)
    line = LineData(l0, TRIPLET)
    psf = None
    route = psf_route(cfg)
    if route is not None and route[0] == "table":
        x, y = gaussian_psf_table(route[1])
        psf = psf_from_table(x, y, offs)
    elif route is not None:
        psf = psf_gaussian(route[1], lam)
    w = Workload(f"config{cfg}", cfg, line, offs, lam, psf, npix or DEFAULT_NPIX[cfg], seed=cfg)
    w.nterms, w.fix, w.guess = nterms_fix_guess(cfg)
    return w


def truth_models(w: Workload, rng: np.random.Generator | None = None) -> np.ndarray:
    """Seeded per-pixel atmospheres [npix][11]."""
    return _truth_models(w.cfg, w.npix, rng or np.random.default_rng(w.seed))


def synthesize(w: Workload, inv_fp64=None, rng: np.random.Generator | None = None, truth: np.ndarray | None = None,
               return_truth: bool = False):
    """Observed profiles [npix][4][nl] float32: FP64 GPU synthesis of the truth
    models plus N(0, 1e-3) noise.  Needs a B200 (the synthesis runs on it)."""
    from . import PREC_FP64, Inverter

    rng = rng or np.random.default_rng(w.seed)
    truth = truth_models(w, rng) if truth is None else truth
    if w.cfg == 2 and w.slight is None:
        with Inverter(w.line, w.lam, w.psf, noise=w.noise, precision=PREC_FP64) as plain:
            w.slight = plain.synth(QUIET_SUN_B0[None, :])[0]
    own = inv_fp64 is None
    if own:
        inv_fp64 = Inverter(w.line, w.lam, w.psf, noise=w.noise, fix=w.fix, nterms=w.nterms, precision=PREC_FP64)
    try:
        obs = inv_fp64.synth(truth, slight=w.slight)
    finally:
        if own:
            inv_fp64.close()
    obs = obs + rng.normal(0.0, NOISE_SIGMA, obs.shape).astype(np.float32)
    obs = np.ascontiguousarray(obs, dtype=np.float32)
    return (obs, truth) if return_truth else obs


def truth_models_device(w: Workload, seed: int, device="cuda"):
    """The truth_models distributions drawn on the device (torch generator
    seeded with ``seed``): for cubes too large to build in host memory."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    n = w.npix

    def U(lo, hi, k=n):
        return lo + (hi - lo) * torch.rand(k, generator=g, device=device, dtype=torch.float64)

    m = torch.zeros((n, 11), dtype=torch.float64, device=device)
    for col, (lo, hi) in enumerate([(1, 20), (0, 3000), (-3, 3), (0.02, 0.05), (0.01, 0.5), (0, 180), (0, 180),
                                    (0.1, 0.4), (0.4, 0.9)]):
        m[:, col] = U(lo, hi)
    m[:, 10] = 1.0
    if w.cfg in (2, 3):
        weak = torch.rand(n, generator=g, device=device) < 0.7
        m[:, 1] = torch.where(weak, U(0, 200), U(1500, 3500))
        m[:, 0] = torch.where(weak, U(1, 5), m[:, 0])
    if w.cfg == 2:
        m[:, 10] = 1.0 - U(0, 0.3)
    return m


def synthesize_device(w: Workload, inv_fp64, seed: int, chunk: int = 1 << 21):
    """Observed profiles as a CUDA float32 tensor [npix][4][nl]: FP64 synthesis
    of device-drawn truth models plus N(0, 1e-3) noise, generated in chunks so
    that only the cube itself (and one chunk of temporaries) is resident."""
    import torch

    truth = truth_models_device(w, seed)
    obs = torch.empty((w.npix, 4, w.nl), dtype=torch.float32, device="cuda")
    g = torch.Generator(device="cuda")
    g.manual_seed(int(seed) + 1)
    for p0 in range(0, w.npix, chunk):
        p1 = min(w.npix, p0 + chunk)
        obs[p0:p1] = inv_fp64.synth(truth[p0:p1], slight=None if w.slight is None else
                                    torch.as_tensor(np.asarray(w.slight, dtype=np.float32), device="cuda"))
        obs[p0:p1] += NOISE_SIGMA * torch.randn((p1 - p0, 4, w.nl), generator=g, device="cuda")
    del truth
    return obs


def psf_support(psf) -> int:
    """Taps the multi-warp correlations use: those above 1e-18 of the peak."""
    if psf is None:
        return 0
    a = np.abs(np.asarray(psf))
    idx = np.nonzero(a > 1e-18 * a.max())[0]
    return int(idx[-1] - idx[0] + 1) if idx.size else 0
