"""Per-pixel wavelength grids (pm_invert_batch_grids / pm_synth_batch_grids).

Every pixel has its own grid: the configuration-1 grid (30 points; 112 points of
tests/golden/ref_cases_wide.npz, 49 points with macroturbulence of
ref_cases_mac.npz for the wide-grid kernels) stretched by up to 1e-3 and shifted
by up to +-20 mA, as a telecentric Fabry-Perot's cavity errors shift it across
the field.  The expected result of a pixel is the oracle's (the reference's, bit
for bit) inversion of that pixel on a single grid equal to its own, with the
context's PSF taps.
"""
import os

import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from conftest import GOLDEN
from gpu_common import LINE_6173, NOISE64, assert_plain_parity, case, within_tolerance

pytestmark = pytest.mark.gpu

CUANTIC = np.array([1.0, *LINE_6173[1]])


def grids(base, n, seed, l0=LINE_6173[0]):
    rng = np.random.default_rng(seed)
    scale = 1.0 + rng.uniform(-1e-3, 1e-3, n)
    shift = rng.uniform(-0.020, 0.020, n)
    return l0 + (base[None, :] - l0) * scale[:, None] + shift[:, None]


def truths(n, seed, mac=False):
    rng = np.random.default_rng(seed)
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
    m[:, 9] = rng.uniform(0.5, 2.5, n) if mac else 0.0
    m[:, 10] = 1.0
    return m


def oracles(lam, psf, nterms):
    return [po.Restatement(po.LineSetup(l, LINE_6173[0], CUANTIC, psf, nterms), "f64") for l in lam]


def fast_models(oras, obs, guess, fix):
    """The reference's own optimised FP64 build on each pixel's grid (None when
    it was not built): the yardstick of gpu_common.assert_plain_parity."""
    if not po.reference_available("f64_fast"):
        return None
    models = [po.Reference(o.setup, "f64_fast").invert(obs[i:i + 1], guess, fix=fix, noise=NOISE64,
                                                        want_spectra=False)["models"] for i, o in enumerate(oras)]
    return {"models": np.concatenate(models)}


def stacked(results):
    return {k: np.concatenate([r[k] for r in results]) for k in ("models", "spectra", "status")}


def observed(oras, models, fix, seed):
    rng = np.random.default_rng(seed)
    obs = np.array([o.synth(m, fix=fix, rf=False)[0] for o, m in zip(oras, models)], dtype=np.float32)
    return obs + rng.normal(0, 1e-3, obs.shape).astype(np.float32)


@pytest.mark.parametrize("mac", [False, True])
def test_synthesis_on_each_pixels_grid(mac):
    c = case(1)
    n = 64
    lam = grids(c["lam"], n, 1)
    nterms, fix = (10, [1] * 10 + [0]) if mac else (9, c["fix"])
    models = truths(n, 2, mac)
    with pm.Inverter(pm.LineData(*LINE_6173), c["lam"], c["psf"], noise=NOISE64, fix=fix, nterms=nterms,
                     precision=pm.PREC_FP64) as inv:
        sp, rf = inv.synth(models, rf=True, lam=lam)
    for o, m, s, r in zip(oracles(lam, c["psf"], nterms), models, sp, rf):
        s_ref, rf_ref = o.synth(m, fix=fix)
        assert np.abs(s - s_ref).max() < 1e-6
        scale = np.abs(rf_ref).max(axis=-1, keepdims=True) + 1e-30
        assert (np.abs(r - rf_ref) / scale).max() < 1e-5


def test_fp64_inversion_on_each_pixels_grid():
    c = case(1)
    n = 96
    lam = grids(c["lam"], n, 3)
    oras = oracles(lam, c["psf"], 9)
    obs = observed(oras, truths(n, 4), c["fix"], 5)
    ref = [o.invert(obs[i:i + 1], c["guess"], fix=c["fix"], noise=NOISE64) for i, o in enumerate(oras)]
    ref_models = np.concatenate([r["models"] for r in ref])
    with pm.Inverter(pm.LineData(*LINE_6173), c["lam"], c["psf"], noise=NOISE64, fix=c["fix"], nterms=9,
                     precision=pm.PREC_FP64, solver=pm.SOLVE_EIGEN) as inv:
        r = inv.invert(obs, c["guess"], lam=lam)
        shared = inv.invert(obs, c["guess"])
    assert_plain_parity(r, stacked(ref), params=tuple(i for i in range(11) if c["fix"][i]),
                        fast=fast_models(oras, obs, c["guess"], c["fix"]))
    # the shifts matter: on the shared grid the same profiles give other models
    assert within_tolerance(shared["models"], ref_models).mean() < 0.5


def test_fp32_inversion_on_each_pixels_grid():
    c = case(1)
    n = 96
    lam = grids(c["lam"], n, 6)
    oras = oracles(lam, c["psf"], 9)
    obs = observed(oras, truths(n, 7), c["fix"], 8)
    ref_models = np.concatenate([o.invert(obs[i:i + 1], c["guess"], fix=c["fix"], noise=NOISE64)["models"]
                                 for i, o in enumerate(oras)])
    with pm.Inverter(pm.LineData(*LINE_6173), c["lam"], c["psf"], noise=NOISE64, fix=c["fix"], nterms=9,
                     precision=pm.PREC_FP32) as inv:
        r = inv.invert(obs, c["guess"], lam=lam)
    dB = np.abs(r["models"][:, 1] - ref_models[:, 1])
    assert np.median(dB) < 1.0
    assert (dB < 5.0).mean() >= 0.9


@pytest.mark.parametrize("prec", [pm.PREC_FP64, pm.PREC_FP32])
def test_identical_grids_give_the_shared_grid_results(prec):
    """Every pixel on the context's own grid: the pixel-grid kernel and the
    shared-grid kernel agree (same arithmetic; the two are separately compiled,
    so within the stated tolerance rather than bit for bit)."""
    c = case(1)
    lam = np.tile(c["lam"], (c["obs"].shape[0], 1))
    with pm.Inverter(pm.LineData(*LINE_6173), c["lam"], c["psf"], noise=NOISE64, fix=c["fix"], nterms=9,
                     precision=prec) as inv:
        a = inv.invert(c["obs"], c["guess"], lam=lam)
        b = inv.invert(c["obs"], c["guess"])
    if prec == pm.PREC_FP64:
        assert within_tolerance(a["models"], b["models"]).all()
    else:
        dB = np.abs(a["models"][:, 1] - b["models"][:, 1])
        assert np.median(dB) < 1.0 and (dB < 5.0).mean() >= 0.9


def test_device_buffers_and_errors():
    import torch

    c = case(1)
    n = c["obs"].shape[0]
    lam = grids(c["lam"], n, 9)
    with pm.Inverter(pm.LineData(*LINE_6173), c["lam"], c["psf"], noise=NOISE64, fix=c["fix"], nterms=9,
                     precision=pm.PREC_FP64) as inv:
        host = inv.invert(c["obs"], c["guess"], lam=lam)
        dev = inv.invert(torch.from_numpy(c["obs"]).cuda(), c["guess"], lam=torch.from_numpy(lam).cuda())
        assert np.array_equal(dev["models"].cpu().numpy(), host["models"])
        assert np.array_equal(dev["iters"].cpu().numpy(), host["iters"])
        with pytest.raises(ValueError):
            inv.invert(c["obs"], c["guess"], lam=lam[:-1])


# ---- grids wider than one warp ----
TRIPLET = (2.0, 1.0, 1.0, 2.0, 2.0, 0.0)


def wide_case(name):
    """w112: the 112-point configuration-4 grid (Fe I 6302.4936, 25 mA PSF, nine
    parameters); mw10: 49 points with v_mac inverted (Fe I 6173.3354, 60 mA PSF)."""
    src = np.load(os.path.join(GOLDEN, "ref_cases_wide.npz" if name == "w112" else "ref_cases_mac.npz"))
    g = lambda k: src[f"{name}_{k}"]
    return dict(lam=g("lam"), l0=float(g("lambda0")), psf=g("psf"), fix=list(g("fix")), nterms=int(g("nterms")),
                guess=g("guess"), mac=name == "mw10")


def wide_inverter(c, precision, solver=pm.SOLVE_DEFAULT):
    return pm.Inverter(pm.LineData(c["l0"], TRIPLET), c["lam"], c["psf"], noise=NOISE64, fix=c["fix"],
                       nterms=c["nterms"], precision=precision, solver=solver)


def wide_oracles(c, lam, flav="f64"):
    return [po.Restatement(po.LineSetup(l, c["l0"], np.array([1.0, *TRIPLET]), c["psf"], c["nterms"]), flav)
            for l in lam]


@pytest.mark.parametrize("name", ["w112", "mw10"])
def test_wide_synthesis_on_each_pixels_grid(name):
    """Two and four warps per pixel: the synthesis and every response function
    (the v_mac row and its kernel, centred on the pixel's own middle wavelength,
    included) on each pixel's grid."""
    c = wide_case(name)
    n = 32
    lam = grids(c["lam"], n, 21, c["l0"])
    models = truths(n, 22, c["mac"])
    with wide_inverter(c, pm.PREC_FP64) as inv:
        sp, rf = inv.synth(models, rf=True, lam=lam)
    for o, m, s_gpu, r_gpu in zip(wide_oracles(c, lam), models, sp, rf):
        s_ref, rf_ref = o.synth(m, fix=c["fix"])
        assert np.abs(s_gpu - s_ref).max() < 1e-6
        scale = np.abs(rf_ref).max(axis=-1, keepdims=True) + 1e-30
        assert (np.abs(r_gpu - rf_ref) / scale).max() < 1e-5


@pytest.mark.parametrize("prec", [pm.PREC_FP64, pm.PREC_FP32])
def test_wide_inversion_on_each_pixels_grid(prec):
    c = wide_case("w112")
    n = 64
    lam = grids(c["lam"], n, 23, c["l0"])
    oras = wide_oracles(c, lam)
    obs = observed(oras, truths(n, 24), c["fix"], 25)
    refs = stacked([o.invert(obs[i:i + 1], c["guess"], fix=c["fix"], noise=NOISE64) for i, o in enumerate(oras)])
    ref = refs["models"]
    with wide_inverter(c, prec, pm.SOLVE_EIGEN if prec == pm.PREC_FP64 else pm.SOLVE_DEFAULT) as inv:
        r = inv.invert(obs, c["guess"], lam=lam)
        shared = inv.invert(obs, c["guess"])
    if prec == pm.PREC_FP64:
        assert_plain_parity(r, refs, params=tuple(i for i in range(11) if c["fix"][i]),
                            fast=fast_models(oras, obs, c["guess"], c["fix"]))
    else:
        dB = np.abs(r["models"][:, 1] - ref[:, 1])
        assert np.median(dB) < 1.0 and (dB < 5.0).mean() >= 0.9
    # the shifts matter: on the shared grid the same profiles give other models
    assert within_tolerance(shared["models"], ref).mean() < 0.5


def test_wide_device_and_host_buffers_agree():
    import torch

    c = wide_case("w112")
    n = 40
    lam = grids(c["lam"], n, 26, c["l0"])
    obs = observed(wide_oracles(c, lam), truths(n, 27), c["fix"], 28)
    with wide_inverter(c, pm.PREC_FP32) as inv:
        host = inv.invert(obs, c["guess"], lam=lam)
        dev = inv.invert(torch.from_numpy(obs).cuda(), c["guess"], lam=torch.from_numpy(lam).cuda())
    for k in ("models", "iters", "chisq"):
        assert np.array_equal(dev[k].cpu().numpy(), host[k]), k
