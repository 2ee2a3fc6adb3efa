"""Shared helpers of the GPU parity tests."""
import os

import numpy as np

import pmilos_b200 as pm
import pyoracle as po
from conftest import GOLDEN

CASES = np.load(os.path.join(GOLDEN, "ref_cases.npz"))
LINE_6173 = (6173.3354, (2.0, 1.0, 1.0, 2.0, 2.0, 0.0))
NOISE64 = (1.0 / 1000) ** 2

# per-parameter tolerances of the plain form against the FP64 oracle (model order)
#   eta0, B, vlos, dopp, aa, gm, az, S0, S1, mac, alfa
ABS_TOL = {1: 1.0, 2: 1e-3, 5: 0.1, 6: 0.1, 9: 1e-3}  # |dB| < 1 G, v, v_mac < 1 m/s, angles < 0.1 deg
REL_TOL = {0: 1e-4, 3: 1e-4, 4: 1e-4, 7: 1e-4, 8: 1e-4, 10: 1e-4}


def case(cfg):
    g = lambda k: CASES[f"c{cfg}_{k}"]
    psf = g("psf") if g("psf").size else None
    sl = g("slight") if g("slight").size else None
    return dict(lam=g("lam"), psf=psf, slight=sl, obs=g("obs"), guess=g("guess"), fix=list(g("fix")),
                nterms=int(g("nterms")), truth=g("truth"))


def inverter(c, precision, solver=pm.SOLVE_DEFAULT, **kw):
    line = pm.LineData(*LINE_6173)
    return pm.Inverter(line, c["lam"], c["psf"], noise=NOISE64, fix=c["fix"], nterms=c["nterms"],
                       precision=precision, solver=solver, **kw)


def oracle(c, flav="f64"):
    return po.Restatement(po.LineSetup(c["lam"], LINE_6173[0], np.array([1.0, *LINE_6173[1]]), c["psf"], c["nterms"]),
                          flav)


def within_tolerance(a, b, params=(0, 1, 2, 3, 4, 5, 6, 7, 8, 10)):
    """Boolean [npix] mask: every listed parameter of a within tolerance of b."""
    ok = np.ones(a.shape[0], dtype=bool)
    for p in params:
        if p in ABS_TOL:
            d = np.abs(a[:, p] - b[:, p])
            if p == 6:  # azimuth is defined modulo 180 deg
                d = np.minimum(d, 180.0 - d)
            ok &= d < ABS_TOL[p]
        else:
            ok &= np.abs(a[:, p] - b[:, p]) <= REL_TOL[p] * np.maximum(np.abs(b[:, p]), 1e-12)
    return ok


# lm_mils' loop ended by one of its own tests (toplim or the damping bound),
# not at the iteration cap: "where both codes converge"
STOPPED = (pm.PIX_CONVERGED, pm.PIX_LAMBDA)


def both_converged(gpu_status, oracle_status):
    """Boolean [npix] mask of the pixels whose LM loop converged in both codes."""
    return np.isin(gpu_status, STOPPED) & np.isin(oracle_status, STOPPED)


def param_error(a, b, p):
    """|a - b| of parameter p per pixel: absolute for the parameters with an
    absolute tolerance (B, v_los, the angles, v_mac; the azimuth modulo 180 deg),
    relative to |b| for the others."""
    d = np.abs(a[:, p] - b[:, p])
    if p == 6:
        d = np.minimum(d, 180.0 - d)
    if p in ABS_TOL:
        return d
    return d / np.maximum(np.abs(b[:, p]), 1e-12)


def reference_fast(setup):
    """The reference's own optimised FP64 build (-O3 -march, oracle/_ref), or None
    when it was not built."""
    return po.Reference(setup, "f64_fast") if po.reference_available("f64_fast") else None


def assert_plain_parity(r, ref, params=(0, 1, 2, 3, 4, 5, 6, 7, 8, 10), fast=None, slack=0.005,
                        min_converged=0.2, spectra_tol=1e-6):
    """The plain form against the FP64 oracle, as the contract states it.

    * Pixels whose loop converges in both codes (the toplim test, PM_PIX_CONVERGED):
      every one within the tolerance, best-fit profiles within spectra_tol I_c.
    * Pixels whose loop stops by either of its tests in both codes (toplim or the
      damping bound): no more outside the tolerance than the reference's own
      optimised build gives against the oracle on the same pixels (``fast``: its
      results, when available) plus ``slack`` of them (at least one) -- a pixel whose chi^2 valley
      is flat along a parameter ends wherever rounding leaves it, in the reference
      as here.
    Returns the mask of pixels within the tolerance."""
    ok = within_tolerance(r["models"], ref["models"], params)
    conv = (r["status"] == pm.PIX_CONVERGED) & (ref["status"] == pm.PIX_CONVERGED)
    assert conv.mean() >= min_converged, f"{conv.mean():.1%} of pixels converged in both codes"
    bad = np.nonzero(conv & ~ok)[0]
    assert bad.size == 0, f"{bad.size} converged pixels outside the tolerance, e.g. {bad[:5]}"
    if "spectra" in r and "spectra" in ref and conv.any():
        ds = float(np.abs(np.asarray(r["spectra"])[conv] - np.asarray(ref["spectra"])[conv]).max())
        assert ds <= spectra_tol, f"best-fit profiles of converged pixels differ by {ds:.2e} I_c"
    stopped = both_converged(r["status"], ref["status"])
    ref_out = 0
    if fast is not None:
        ref_out = int((np.isin(ref["status"], STOPPED) & ~within_tolerance(fast["models"], ref["models"], params)).sum())
    gpu_out = int((stopped & ~ok).sum())
    assert gpu_out <= ref_out + max(1.0, slack * stopped.sum()), \
        f"{gpu_out} stopped pixels outside the tolerance; the reference's own builds differ on {ref_out}"
    return ok
