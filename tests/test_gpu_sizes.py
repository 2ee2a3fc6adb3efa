"""Grid sizes at the edges of the kernels' layouts.

3 wavelengths (the fewest with degrees of freedom for nine parameters), odd and
even sizes inside one warp, 32 (a full warp, no idle lane), 33 and 64 (two warps
per pixel, one lane of the second in use / both full), 65 and 128 (four warps,
the largest grid), with a 60 mA Gaussian PSF sampled on each grid (odd sizes
move the PSF centre tap).  FP64 synthesis, response functions and inversions
against the FP64 oracle; 129 wavelengths are refused.
"""
import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from gpu_common import LINE_6173, NOISE64, within_tolerance

pytestmark = pytest.mark.gpu

SIZES = [3, 7, 17, 31, 32, 33, 47, 64, 65, 100, 127, 128]
FIX = [1] * 9 + [0, 0]
GUESS = np.array([8.0, 400.0, 0.0, 0.03, 0.1, 30.0, 30.0, 0.25, 0.75, 0.0, 1.0])


def grid(nl):
    # a span of about 0.7 A whatever the size: a few points straddle the line
    step = 0.7 / max(nl - 1, 1)
    return LINE_6173[0] + (np.arange(nl) - nl // 2) * step + 0.003


def models(n, seed):
    rng = np.random.default_rng(seed)
    m = np.zeros((n, 11))
    m[:, 0] = rng.uniform(2, 20, n)
    m[:, 1] = rng.uniform(100, 2500, n)
    m[:, 2] = rng.uniform(-2, 2, n)
    m[:, 3] = rng.uniform(0.025, 0.045, n)
    m[:, 4] = rng.uniform(0.02, 0.4, n)
    m[:, 5] = rng.uniform(10, 170, n)
    m[:, 6] = rng.uniform(10, 170, n)
    m[:, 7] = rng.uniform(0.1, 0.4, n)
    m[:, 8] = rng.uniform(0.4, 0.9, n)
    m[:, 10] = 1.0
    return m


def setup(nl):
    lam = grid(nl)
    psf = pm.psf_gaussian(60.0, lam)
    ora = po.Restatement(po.LineSetup(lam, LINE_6173[0], np.array([1.0, *LINE_6173[1]]), psf, 9), "f64")
    inv = pm.Inverter(pm.LineData(*LINE_6173), lam, psf, noise=NOISE64, fix=FIX, nterms=9, precision=pm.PREC_FP64,
                      solver=pm.SOLVE_EIGEN)
    return lam, psf, ora, inv


@pytest.mark.parametrize("nl", SIZES)
def test_synthesis_and_rf_at_the_edges(nl):
    _, _, ora, inv = setup(nl)
    m = models(24, nl)
    with inv:
        sp, rf = inv.synth(m, rf=True)
    for i in range(m.shape[0]):
        s_ref, rf_ref = ora.synth(m[i], fix=FIX)
        assert np.abs(sp[i] - s_ref).max() < 1e-6, i
        scale = np.abs(rf_ref).max(axis=-1, keepdims=True) + 1e-30
        assert (np.abs(rf[i] - rf_ref) / scale).max() < 1e-5, i


@pytest.mark.parametrize("nl", [7, 32, 33, 64, 65, 128])
def test_inversion_at_the_edges(nl):
    _, _, ora, inv = setup(nl)
    truth = models(48, 100 + nl)
    rng = np.random.default_rng(nl)
    obs = np.array([ora.synth(t, fix=FIX, rf=False)[0] for t in truth], dtype=np.float32)
    obs += rng.normal(0, 1e-3, obs.shape).astype(np.float32)
    ref = ora.invert(obs, GUESS, fix=FIX, noise=NOISE64)
    with inv:
        r = inv.invert(obs, GUESS)
    ok = within_tolerance(r["models"], ref["models"])
    assert ok.mean() >= 0.8, f"only {ok.mean():.2%} of pixels within tolerance"
    assert np.abs(r["spectra"][ok] - ref["spectra"][ok]).max() < 1e-5
    # iteration counts follow rounding (the reference's own pin and fast builds
    # agree on them for only a third to most of the pixels): medians within 15%
    assert abs(np.median(r["iters"]) - np.median(ref["iters"])) <= max(3.0, 0.15 * np.median(ref["iters"]))


def test_grid_too_wide_is_refused():
    lam = grid(129)
    with pytest.raises(pm.PmError) as e:
        pm.Inverter(pm.LineData(*LINE_6173), lam, None, noise=NOISE64, fix=FIX, nterms=9)
    assert e.value.code == -34  # PM_ERANGE
