"""The stated tolerances, free parameter by free parameter, on the grid of every
benchmark configuration.

Cubes: 2048 pixels (1024 on the 112-point grid) drawn from each configuration's
distributions (seeded), profiles synthesized by the FP64 oracle, N(0, 1e-3)
noise; configuration 3 on each of its three grids (6, 15 and 30 points, the
numeric-FWHM PSF route).  How lm_mils' loop ended is compared pixel by pixel
(milosUtils.c:600-630): by its convergence test (toplim: chi^2 no longer
changes, PM_PIX_CONVERGED), by the damping bound (seven rejected steps in a row,
PM_PIX_LAMBDA), or at the iteration cap.

* Plain form (FP64, eigen solve) against the FP64 oracle:
  - on the pixels where both codes converge (PM_PIX_CONVERGED in both): every
    one within |dB| < 1 G, angles < 0.1 deg, v_los < 1 m/s and 1e-4 relative for
    the other parameters, and best-fit profiles within 1e-6 I_c;
  - on the pixels where both loops stop by one of their tests (either status):
    no more pixels outside that tolerance than the reference's own two FP64
    builds (-O2 and -O3 -march, the oracle's bit-exact twin and the optimised
    build) give on the same pixels, plus 0.5% -- a pixel whose valley is flat
    along some parameter (the azimuth of a nearly longitudinal field, most
    parameters on the 6-point grid) ends wherever rounding leaves it, in the
    reference as here.
* Batched form (FP32 synthesis, response functions, convolution and normal
  equations; FP64 solve and acceptance test) against the FP64 oracle, on the
  pixels where both stop by one of their tests (for the inclination, those with
  B >= 100 G; for the azimuth, a transverse field >= 100 G: below that the field
  does not define the angle): the 99th percentile of each parameter's error
  within FP32_TOL[configuration], and, on the grids that sample
  the line (15 to 112 points), within twice the reference float build's own 99th
  percentile on the same pixels (the reference's default REAL = float, the
  precision it ships with) plus a floor.  On the 6-point grid (24 data for 9
  parameters, no sample at the line centre) the float build is the more accurate
  one -- its Voigt function runs in double inside (fvoigt.c:15-80) -- and the
  FP32 form's stated tolerance there is correspondingly loose (_SIX).
* The fraction of pixels that stop by a test is bounded below, so that no bar
  can pass on a handful of pixels.
"""
import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from gpu_common import NOISE64, STOPPED, both_converged, param_error, within_tolerance
from pmilos_b200 import workloads

pytestmark = pytest.mark.gpu

# (configuration, grid of configuration 3, pixels)
CASES = [(1, 2, 2048), (2, 2, 2048), (3, 0, 2048), (3, 1, 2048), (3, 2, 2048), (4, 2, 1024)]
IDS = ["c1", "c2", "c3-6pt", "c3-15pt", "c3-30pt", "c4-112pt"]

# The stated FP32 tolerance against the FP64 oracle: the 99th percentile of each
# parameter's error over the pixels where both loops stop by a test; absolute
# for B [G], v_los [km/s] and the angles [deg], relative for the others.  One
# table for the grids that sample the line (15 to 112 points), one for the
# 6-point grid, which has no sample at the line centre and 24 data for 9
# parameters.
_SAMPLED = {0: 5e-2, 1: 0.5, 2: 2e-4, 3: 5e-3, 4: 1e-2, 5: 0.1, 6: 1.0, 7: 5e-2, 8: 2e-2, 10: 1e-4}
_SIX = {0: 0.3, 1: 200.0, 2: 0.3, 3: 0.6, 4: 0.05, 5: 1.0, 6: 40.0, 7: 0.06, 8: 0.02}
FP32_TOL = {"c1": _SAMPLED, "c2": _SAMPLED, "c3-6pt": _SIX, "c3-15pt": _SAMPLED, "c3-30pt": _SAMPLED,
            "c4-112pt": _SAMPLED}
FP32_QUANTILE = 0.99
# lower bounds of the fraction of pixels whose loop stops by a test in both codes
MIN_STOPPED = {"c1": 0.75, "c2": 0.35, "c3-6pt": 0.25, "c3-15pt": 0.5, "c3-30pt": 0.4, "c4-112pt": 0.85}
MIN_CONVERGED = {"c1": 0.6, "c2": 0.3, "c3-6pt": 0.15, "c3-15pt": 0.4, "c3-30pt": 0.35, "c4-112pt": 0.75}

_CACHE = {}


def _setup(w):
    return po.LineSetup(w.lam, w.line.lambda0, w.line.cuantic_dat(), w.psf, w.nterms)


def _cube(cfg, grid, npix):
    key = (cfg, grid, npix)
    if key in _CACHE:
        return _CACHE[key]
    w = workloads.config(cfg, npix=npix, grid=grid)
    ora = po.Restatement(_setup(w), "f64")
    rng = np.random.default_rng(70 + 10 * cfg + grid)
    truth = workloads.truth_models(w, rng)
    sl = None
    if cfg == 2:  # the stray-light profile: a B = 0 quiet-Sun atmosphere, as float32
        s9 = po.LineSetup(w.lam, w.line.lambda0, w.line.cuantic_dat(), w.psf, 9)
        sl = po.Restatement(s9, "f64").synth(workloads.QUIET_SUN_B0, rf=False)[0]
        sl = sl.astype(np.float32).astype(np.float64)
    obs = np.array([ora.synth(m, sl, fix=w.fix, rf=False)[0] for m in truth], dtype=np.float32)
    obs += rng.normal(0, 1e-3, obs.shape).astype(np.float32)
    ref = ora.invert(obs, w.guess, slight=sl, fix=w.fix, noise=NOISE64)
    _CACHE[key] = (w, obs, sl, ref)
    return _CACHE[key]


def _invert(w, obs, sl, precision, solver=pm.SOLVE_DEFAULT):
    slf = None if sl is None else sl.astype(np.float32)
    with pm.Inverter(w.line, w.lam, w.psf, noise=NOISE64, fix=w.fix, nterms=w.nterms, precision=precision,
                     solver=solver) as inv:
        return inv.invert(obs, w.guess, slight=slf)


def _free(w):
    return tuple(i for i in range(11) if w.fix[i])


def _name(cfg, grid, npix):
    return IDS[CASES.index((cfg, grid, npix))]


@pytest.mark.parametrize("cfg,grid,npix", CASES, ids=IDS)
def test_plain_form_meets_the_stated_tolerance_where_both_converge(cfg, grid, npix):
    w, obs, sl, ref = _cube(cfg, grid, npix)
    name = _name(cfg, grid, npix)
    r = _invert(w, obs, sl, pm.PREC_FP64, pm.SOLVE_EIGEN)
    ok = within_tolerance(r["models"], ref["models"], _free(w))
    conv = (r["status"] == pm.PIX_CONVERGED) & (ref["status"] == pm.PIX_CONVERGED)
    assert conv.mean() >= MIN_CONVERGED[name], f"{conv.mean():.1%} of pixels converged in both codes"
    bad = np.nonzero(conv & ~ok)[0]
    assert bad.size == 0, f"{bad.size} converged pixels outside the tolerance, e.g. {bad[:5]}"
    dspec = np.abs(r["spectra"][conv] - ref["spectra"][conv]).max()
    assert dspec <= 1e-6, f"best-fit profiles differ by {dspec:.2e} I_c"
    # every pixel that stops by a test: no more outliers than the reference's own builds give
    stopped = both_converged(r["status"], ref["status"])
    assert stopped.mean() >= MIN_STOPPED[name], f"{stopped.mean():.1%} of pixels stopped by a test in both codes"
    fast = po.Reference(_setup(w), "f64_fast").invert(obs, w.guess, slight=sl, fix=w.fix, noise=NOISE64,
                                                     want_spectra=False)
    ref_out = int((np.isin(ref["status"], STOPPED) & ~within_tolerance(fast["models"], ref["models"], _free(w))).sum())
    gpu_out = int((stopped & ~ok).sum())
    assert gpu_out <= ref_out + 0.005 * stopped.sum(), (gpu_out, ref_out, int(stopped.sum()))


@pytest.mark.parametrize("cfg,grid,npix", CASES, ids=IDS)
def test_fp32_form_meets_its_stated_tolerance_where_both_converge(cfg, grid, npix):
    w, obs, sl, ref = _cube(cfg, grid, npix)
    name = _name(cfg, grid, npix)
    r = _invert(w, obs, sl, pm.PREC_FP32)
    stopped = both_converged(r["status"], ref["status"])
    assert stopped.mean() >= MIN_STOPPED[name], f"{stopped.mean():.1%} of pixels stopped by a test in both codes"
    # the reference's float build on the same pixels: the precision it ships with
    f32 = po.Restatement(_setup(w), "f32").invert(obs, w.guess, slight=sl, fix=w.fix,
                                                  noise=float(np.float32(np.float32(1e-3) ** 2)), want_spectra=False)
    both_f32 = stopped & np.isin(f32["status"], STOPPED)
    # the angles where the field defines them (the oracle's B >= 100 G for the
    # inclination, its transverse component >= 100 G for the azimuth)
    B, gm = ref["models"][:, 1], np.radians(ref["models"][:, 5])
    defined = {5: B >= 100.0, 6: B * np.abs(np.sin(gm)) >= 100.0}
    for p in _free(w):
        sel = stopped & defined.get(p, True)
        q = np.quantile(param_error(r["models"], ref["models"], p)[sel], FP32_QUANTILE)
        assert q <= FP32_TOL[name][p], f"{pm.MODEL_FIELDS[p]}: {FP32_QUANTILE:.0%} quantile {q:.3g} > {FP32_TOL[name][p]}"
        if name == "c3-6pt":
            continue  # see the module docstring: the float build's FP64 Voigt function matters on this grid
        sel32 = both_f32 & defined.get(p, True)
        q_here = np.quantile(param_error(r["models"], ref["models"], p)[sel32], FP32_QUANTILE)
        q_ref = np.quantile(param_error(f32["models"], ref["models"], p)[sel32], FP32_QUANTILE)
        floor = 0.1 * FP32_TOL["c1"][p]
        assert q_here <= 2 * q_ref + floor, f"{pm.MODEL_FIELDS[p]}: {q_here:.3g} against the float build's {q_ref:.3g}"
    assert np.isfinite(r["models"]).all() and np.all(r["status"] >= 0)
