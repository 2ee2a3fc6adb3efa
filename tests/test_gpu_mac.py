"""Macroturbulence on the GPU (one warp per pixel, 30 wavelengths).

Cases from tests/golden/ref_cases_mac.npz (made by running the reference): m10
(v_mac inverted, 60 mA PSF), m10n (the same without PSF), m11 (v_mac and the
filling factor inverted, stray light), mfix (v_mac fixed at 1.2 km/s, NTERMS 10)
on the 30-point grid; mw10 (as m10 on 49 points: two warps per pixel) and mw11
(as m11 on 112 points: four warps per pixel), whose inversions add 40 pixels
synthesized by the FP64 oracle with N(0, 1e-3) noise to the fixture's 16.
The GPU is compared with the FP64 oracle restatement, which equals the reference
bit for bit on these cases (tests/test_oracle_pin.py).
"""
import os

import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from conftest import GOLDEN
from gpu_common import LINE_6173, NOISE64, assert_plain_parity, reference_fast, within_tolerance

pytestmark = pytest.mark.gpu

MAC = np.load(os.path.join(GOLDEN, "ref_cases_mac.npz"))
NAMES = ["m10", "m10n", "m11", "mfix", "mw10", "mw11"]
STEP = np.array([0.1, 10.0, 0.01, 1e-3, 1e-2, 1.0, 1.0, 1e-2, 1e-2, 1e-2, 1e-2])
PARAMS = (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10)


def mcase(name):
    g = lambda k: MAC[f"{name}_{k}"]
    return dict(lam=g("lam"), psf=g("psf") if g("psf").size else None,
                slight=g("slight") if g("slight").size else None, obs=g("obs"), guess=g("guess"),
                fix=list(g("fix")), nterms=int(g("nterms")), truth=g("truth"), models=g("f64_synth_models"))


def minverter(c, precision, solver=pm.SOLVE_DEFAULT):
    return pm.Inverter(pm.LineData(*LINE_6173), c["lam"], c["psf"], noise=NOISE64, fix=c["fix"],
                       nterms=c["nterms"], precision=precision, solver=solver)


def moracle(c, flav="f64"):
    return po.Restatement(po.LineSetup(c["lam"], LINE_6173[0], np.array([1.0, *LINE_6173[1]]), c["psf"],
                                       c["nterms"]), flav)


def _models(c, n, seed):
    """Fresh models around the fixture's, v_mac in [0.3, 3] km/s."""
    rng = np.random.default_rng(seed)
    m = np.repeat(c["models"][:1], n, axis=0)
    m[:, 0] = rng.uniform(1, 20, n)
    m[:, 1] = rng.uniform(0, 3000, n)
    m[:, 2] = rng.uniform(-3, 3, n)
    m[:, 3] = rng.uniform(0.02, 0.05, n)
    m[:, 4] = rng.uniform(0.01, 0.5, n)
    m[:, 5] = rng.uniform(0, 180, n)
    m[:, 6] = rng.uniform(0, 180, n)
    m[:, 9] = rng.uniform(0.3, 3.0, n)
    if c["slight"] is not None:
        m[:, 10] = rng.uniform(0.7, 1.0, n)
    return np.concatenate([c["models"], m])


def _observed(c, name, seed):
    """The fixture's profiles, and on the wide grids 40 more from fresh models."""
    if not name.startswith("mw"):
        return c["obs"]
    rng = np.random.default_rng(seed)
    ora = moracle(c)
    extra = np.array([ora.synth(m, c["slight"], fix=c["fix"], rf=False)[0] for m in _models(c, 40, seed)[-40:]],
                     dtype=np.float32)
    extra += rng.normal(0, 1e-3, extra.shape).astype(np.float32)
    return np.concatenate([c["obs"], extra])


@pytest.mark.parametrize("name", NAMES)
def test_fp64_synthesis_and_rf_match_oracle(name):
    """Synthesis and every response function (the v_mac row included) in FP64."""
    c = mcase(name)
    models = _models(c, 40, 11)
    with minverter(c, pm.PREC_FP64) as inv:
        sp, rf = inv.synth(models, slight=c["slight"], rf=True)
    ora = moracle(c)
    for i in range(models.shape[0]):
        s_ref, rf_ref = ora.synth(models[i], c["slight"], fix=c["fix"])
        assert np.abs(sp[i] - s_ref).max() < 1e-6
        scale = np.abs(rf_ref).max(axis=-1, keepdims=True) + 1e-30
        assert (np.abs(rf[i] - rf_ref) / scale).max() < 1e-5, i


@pytest.mark.parametrize("name", ["m10", "m11", "mw11"])
def test_fp32_synthesis_close_to_fp64_oracle(name):
    """The FP32 criterion of the other grids: profiles within 2e-6 of FP64, each
    response function no worse than the reference's own float build, or within
    1% of its row maximum, or within 1e-6 over a typical step."""
    c = mcase(name)
    models = _models(c, 40, 12)
    with minverter(c, pm.PREC_FP32) as inv:
        sp, rf = inv.synth(models, slight=c["slight"], rf=True)
    o64, o32 = moracle(c, "f64"), moracle(c, "f32")
    worst = 0.0
    for i in range(models.shape[0]):
        s_ref, rf_ref = o64.synth(models[i], c["slight"], fix=c["fix"])
        _, rf_r32 = o32.synth(models[i], c["slight"], fix=c["fix"])
        worst = max(worst, np.abs(sp[i] - s_ref).max())
        rowmax = np.abs(rf_ref).max(axis=-1)
        e_gpu = np.abs(rf[i] - rf_ref).max(axis=-1)
        e_r32 = np.abs(rf_r32 - rf_ref).max(axis=-1)
        floor = 1e-6 / STEP[: rf_ref.shape[1]][None, :]
        assert np.all(e_gpu <= np.maximum(np.maximum(2.0 * e_r32, 1e-2 * rowmax), floor))
    assert worst < 2e-6


@pytest.mark.parametrize("name", ["m10", "mw10"])
def test_vanishing_vmac_falls_back_to_the_psf(name):
    """v_mac <= 1e-4: no broadening, the PSF correlation with the continuum
    padding of Stokes I instead -- the profiles of an NTERMS-9 context.  The
    v_mac row is zero then (the reference leaves the previous call's row in
    place; this implementation keeps no state between pixels)."""
    c = mcase(name)
    models = _models(c, 16, 13)
    models[::2, 9] = 0.0
    models[1::2, 9] = 5e-5
    with minverter(c, pm.PREC_FP64) as inv:
        sp, rf = inv.synth(models, rf=True)
    fix9 = [1] * 9 + [0, 0]
    with pm.Inverter(pm.LineData(*LINE_6173), c["lam"], c["psf"], noise=NOISE64, fix=fix9, nterms=9,
                     precision=pm.PREC_FP64) as inv9:
        sp9, rf9 = inv9.synth(models, rf=True)
    assert np.abs(sp - sp9).max() < 1e-12
    scale = np.abs(rf9).max(axis=-1, keepdims=True) + 1e-30
    assert (np.abs(rf[:, :, :9] - rf9) / scale).max() < 1e-10
    assert np.all(rf[:, :, 9] == 0)


@pytest.mark.parametrize("name", ["m10", "mw10"])
@pytest.mark.parametrize("prec", [pm.PREC_FP64, pm.PREC_FP32])
def test_pixel_results_do_not_depend_on_the_warps_history(prec, name):
    """Warps take pixel after pixel; a pixel with v_mac > 1e-4 leaves its data in
    the rows the PSF correlation of the next one pads with zeros.  Synthesis:
    a batch larger than the grid's warps with broadened and unbroadened models
    mixed at random equals the two kinds synthesized apart.  Inversion: 400
    copies of the fixture cube, taken by the persistent kernel's warps (the wide
    kernel's blocks) in whatever order, all give the results of the first copy."""
    c = mcase(name)
    rng = np.random.default_rng(14)
    models = _models(c, 24000, 15)
    off = rng.random(models.shape[0]) < 0.5
    models[off, 9] = 0.0
    with minverter(c, prec) as inv:
        sp, rf = inv.synth(models, rf=True)
        sp_on, rf_on = inv.synth(models[~off], rf=True)
        sp_off, rf_off = inv.synth(models[off], rf=True)
        assert np.array_equal(sp[~off], sp_on) and np.array_equal(rf[~off], rf_on)
        assert np.array_equal(sp[off], sp_off) and np.array_equal(rf[off], rf_off)
        n = c["obs"].shape[0]
        r = inv.invert(np.tile(c["obs"], (400, 1, 1)), c["guess"])
    for k in ("models", "chisq", "iters", "spectra"):
        first = r[k][:n]
        assert np.array_equal(r[k].reshape(400, n, *first.shape[1:]), np.broadcast_to(first, (400, *first.shape))), k


@pytest.mark.parametrize("name", NAMES)
def test_plain_fp64_inversion_matches_oracle(name):
    c = mcase(name)
    obs = _observed(c, name, 62)
    ref = moracle(c).invert(obs, c["guess"], slight=c["slight"], fix=c["fix"], noise=NOISE64)
    with minverter(c, pm.PREC_FP64, pm.SOLVE_EIGEN) as inv:
        r = inv.invert(obs, c["guess"], slight=c["slight"])
    fast = reference_fast(po.LineSetup(c["lam"], LINE_6173[0], np.array([1.0, *LINE_6173[1]]), c["psf"],
                                       c["nterms"]))
    fast_r = None if fast is None else fast.invert(obs, c["guess"], slight=c["slight"], fix=c["fix"],
                                                   noise=NOISE64, want_spectra=False)
    free = tuple(i for i in PARAMS if c["fix"][i])
    ok = assert_plain_parity(r, ref, params=free, fast=fast_r, min_converged=0.1)
    # best-fit profiles where the models agree: most pixels stop at the
    # iteration limit, where two summation orders can part inside the tolerance
    ds = np.abs(r["spectra"] - ref["spectra"]).max(axis=(1, 2))[ok]
    assert np.quantile(ds, 0.9) < 1e-5 and ds.max() < 1e-4
    assert np.allclose(np.sort(r["chisq"][ok]), np.sort(ref["chisq"][ok]), rtol=1e-3)
    assert abs(np.median(r["iters"]) - np.median(ref["iters"])) <= 2
    if c["fix"][9] == 0:
        assert np.all(r["models"][:, 9] == c["guess"][9])


@pytest.mark.parametrize("name", ["m10", "m11", "mw10", "mw11"])
def test_fp32_inversion_against_fp64_oracle(name):
    c = mcase(name)
    obs = _observed(c, name, 63)
    ref = moracle(c).invert(obs, c["guess"], slight=c["slight"], fix=c["fix"], noise=NOISE64)
    with minverter(c, pm.PREC_FP32) as inv:
        r = inv.invert(obs, c["guess"], slight=c["slight"])
    # the stated FP32 tolerance: |dB| < 5 G for 90% of pixels, median below 1 G
    dB = np.abs(r["models"][:, 1] - ref["models"][:, 1])
    assert np.median(dB) < 1.0
    assert (dB < 5.0).mean() >= 0.9
    dmac = np.abs(r["models"][:, 9] - ref["models"][:, 9])
    assert np.median(dmac) < 1e-2
    assert np.all(r["status"] >= 0)


def test_nterms_must_follow_the_guess():
    """NTERMS = 11 - !fix[10] - (v_mac == 0 && !fix[9]) (milos.c:152-157)."""
    c = mcase("mfix")
    with minverter(c, pm.PREC_FP64) as inv:  # NTERMS 10 with v_mac fixed at 1.2
        g = c["guess"].copy()
        g[9] = 0.0
        with pytest.raises(pm.PmError) as e:
            inv.invert(c["obs"][:4], g)
        assert e.value.code == -22  # PM_EINVAL
