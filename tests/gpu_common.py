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
