"""A Zeeman multiplet on the GPU: Fe I 6301.5012 (5P2.0-5D2.0; five pi and four
sigma components per group), from tests/golden/ref_cases_zeeman.npz (made by
running the reference), 60 mA PSF: z9 (30 wavelengths, nine parameters), z10
(30 wavelengths, stray light, filling factor inverted), zw9 (49 wavelengths: two
warps per pixel), zw10 (112 wavelengths, four warps per pixel, stray light), and
with v_mac inverted zm10 (30 wavelengths) and zmw11 (112 wavelengths, stray
light, filling factor inverted).
The oracle equals the reference bit for bit on these cases
(tests/test_oracle_pin.py).  Inversions run on the fixture's pixels plus 40
pixels synthesized by the FP64 oracle with N(0, 1e-3) noise.
"""
import os

import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from conftest import GOLDEN
from gpu_common import NOISE64, assert_plain_parity, reference_fast, within_tolerance

pytestmark = pytest.mark.gpu

ZEE = np.load(os.path.join(GOLDEN, "ref_cases_zeeman.npz"))
NAMES = ["z9", "z10", "zw9", "zw10", "zm10", "zmw11"]
LINE = pm.LineData(6301.5012, (2.0, 1.0, 2.0, 2.0, 2.0, 2.0))
STEP = np.array([0.1, 10.0, 0.01, 1e-3, 1e-2, 1.0, 1.0, 1e-2, 1e-2, 1e-2, 1e-2])
NOISE32 = float(np.float32(np.float32(1e-3) ** 2))  # the float build's 1/SN^2


def zcase(name):
    g = lambda k: ZEE[f"{name}_{k}"]
    return dict(lam=g("lam"), psf=g("psf"), slight=g("slight") if g("slight").size else None, obs=g("obs"),
                guess=g("guess"), fix=list(g("fix")), nterms=int(g("nterms")), cuantic=g("cuantic"),
                models=g("f64_synth_models"))


def zinv(c, precision, solver=pm.SOLVE_DEFAULT):
    return pm.Inverter(LINE, c["lam"], c["psf"], noise=NOISE64, fix=c["fix"], nterms=c["nterms"],
                       precision=precision, solver=solver)


def zora(c, flav="f64"):
    return po.Restatement(po.LineSetup(c["lam"], LINE.lambda0, c["cuantic"], c["psf"], c["nterms"]), flav)


def _models(c, n, seed):
    rng = np.random.default_rng(seed)
    m = np.repeat(c["models"][:1], n, axis=0)
    m[:, 0] = rng.uniform(1, 20, n)
    m[:, 1] = rng.uniform(0, 3000, n)
    m[:, 2] = rng.uniform(-3, 3, n)
    m[:, 3] = rng.uniform(0.02, 0.05, n)
    m[:, 4] = rng.uniform(0.01, 0.5, n)
    m[:, 5] = rng.uniform(0, 180, n)
    m[:, 6] = rng.uniform(0, 180, n)
    if c["slight"] is not None:
        m[:, 10] = rng.uniform(0.7, 1.0, n)
    if c["fix"][9]:
        m[:, 9] = rng.uniform(0.3, 3.0, n)
    return np.concatenate([c["models"], m])


def _params(c):
    """The parameters compared: v_mac too where it is inverted."""
    return tuple(range(11)) if c["fix"][9] else (0, 1, 2, 3, 4, 5, 6, 7, 8, 10)


def _observed(c, seed):
    """The fixture's profiles and 40 more from fresh models, as float32."""
    rng = np.random.default_rng(seed)
    ora = zora(c)
    extra = np.array([ora.synth(m, c["slight"], fix=c["fix"], rf=False)[0] for m in _models(c, 40, seed)[-40:]],
                     dtype=np.float32)
    extra += rng.normal(0, 1e-3, extra.shape).astype(np.float32)
    return np.concatenate([c["obs"], extra])


@pytest.mark.parametrize("name", NAMES)
def test_fp64_synthesis_and_rf_match_oracle(name):
    c = zcase(name)
    models = _models(c, 40, 21)
    with zinv(c, pm.PREC_FP64) as inv:
        sp, rf = inv.synth(models, slight=c["slight"], rf=True)
    ora = zora(c)
    for i in range(models.shape[0]):
        s_ref, rf_ref = ora.synth(models[i], c["slight"], fix=c["fix"])
        assert np.abs(sp[i] - s_ref).max() < 1e-6
        scale = np.abs(rf_ref).max(axis=-1, keepdims=True) + 1e-30
        assert (np.abs(rf[i] - rf_ref) / scale).max() < 1e-5, i


@pytest.mark.parametrize("name", ["z9", "zw10", "zm10", "zmw11"])
def test_fp32_synthesis_close_to_fp64_oracle(name):
    """The FP32 criterion of the other lines: profiles within 2e-6 of FP64, each
    response function no worse than the reference's own float build, or within
    1% of its row maximum, or within 1e-6 over a typical step."""
    c = zcase(name)
    models = _models(c, 40, 22)
    with zinv(c, pm.PREC_FP32) as inv:
        sp, rf = inv.synth(models, slight=c["slight"], rf=True)
    o64, o32 = zora(c, "f64"), zora(c, "f32")
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


@pytest.mark.parametrize("name", NAMES)
def test_plain_fp64_inversion_matches_oracle(name):
    c = zcase(name)
    obs = _observed(c, 31)
    ref = zora(c).invert(obs, c["guess"], slight=c["slight"], fix=c["fix"], noise=NOISE64)
    with zinv(c, pm.PREC_FP64, pm.SOLVE_EIGEN) as inv:
        r = inv.invert(obs, c["guess"], slight=c["slight"])
    fast = reference_fast(po.LineSetup(c["lam"], LINE.lambda0, c["cuantic"], c["psf"], c["nterms"]))
    fast_r = None if fast is None else fast.invert(obs, c["guess"], slight=c["slight"], fix=c["fix"],
                                                   noise=NOISE64, want_spectra=False)
    ok = assert_plain_parity(r, ref, params=_params(c), fast=fast_r, min_converged=0.0)
    # the best-fit profiles are the last trial model's, as lm_mils returns them
    # (not always the returned model's); most multiplet pixels stop at the
    # iteration limit, and where the models agree the reference's own pin and
    # fast builds differ by up to 6e-5 here (1e-9 at the 90th percentile)
    ds = np.abs(r["spectra"] - ref["spectra"]).max(axis=(1, 2))[ok]
    assert np.quantile(ds, 0.9) < 1e-5 and ds.max() < 1e-4
    assert abs(np.median(r["iters"]) - np.median(ref["iters"])) <= 3


def _fp32_bar(dB_ref32):
    """|dB| < 5 G for 90% of pixels less a 5% margin, lowered to what the
    reference's own float build (REAL = float, the oracle's bit-exact
    restatement) reaches on the same pixels when that is less."""
    return min(0.9, float((dB_ref32 < 5.0).mean())) - 0.05


@pytest.mark.parametrize("name", NAMES)
def test_fp32_inversion_against_fp64_oracle(name):
    c = zcase(name)
    obs = _observed(c, 32)
    ref = zora(c).invert(obs, c["guess"], slight=c["slight"], fix=c["fix"], noise=NOISE64)
    r32 = zora(c, "f32").invert(obs, c["guess"], slight=c["slight"], fix=c["fix"], noise=NOISE32)
    with zinv(c, pm.PREC_FP32) as inv:
        r = inv.invert(obs, c["guess"], slight=c["slight"])
    dB = np.abs(r["models"][:, 1] - ref["models"][:, 1])
    assert np.median(dB) < 1.0
    assert (dB < 5.0).mean() >= _fp32_bar(np.abs(r32["models"][:, 1] - ref["models"][:, 1]))
    assert np.all(r["status"] >= 0)


def _pixel_grids(base, n, seed):
    """The grid stretched by up to 1e-3 and shifted by up to +-20 mA per pixel."""
    rng = np.random.default_rng(seed)
    l0 = LINE.lambda0
    scale = 1.0 + rng.uniform(-1e-3, 1e-3, n)
    shift = rng.uniform(-0.020, 0.020, n)
    return l0 + (base[None, :] - l0) * scale[:, None] + shift[:, None]


def test_multiplet_on_each_pixels_grid():
    """Per-pixel wavelength grids with the multiplet: synthesis and the FP64
    inversion of every pixel against the oracle on the pixel's own grid (with the
    context's PSF taps), the FP32 inversion within the stated tolerance."""
    c = zcase("z9")
    n = 48
    lam = _pixel_grids(c["lam"], n, 41)
    oras = [po.Restatement(po.LineSetup(l, LINE.lambda0, c["cuantic"], c["psf"], 9), "f64") for l in lam]
    models = _models(c, n, 42)[-n:]
    with zinv(c, pm.PREC_FP64) as inv:
        sp, rf = inv.synth(models, rf=True, lam=lam)
    for o, m, s_gpu, r_gpu in zip(oras, models, sp, rf):
        s_ref, rf_ref = o.synth(m, fix=c["fix"])
        assert np.abs(s_gpu - s_ref).max() < 1e-6
        scale = np.abs(rf_ref).max(axis=-1, keepdims=True) + 1e-30
        assert (np.abs(r_gpu - rf_ref) / scale).max() < 1e-5
    rng = np.random.default_rng(43)
    obs = np.array([o.synth(m, fix=c["fix"], rf=False)[0] for o, m in zip(oras, models)], dtype=np.float32)
    obs += rng.normal(0, 1e-3, obs.shape).astype(np.float32)
    refs = [o.invert(obs[i:i + 1], c["guess"], fix=c["fix"], noise=NOISE64) for i, o in enumerate(oras)]
    refs = {k: np.concatenate([x[k] for x in refs]) for k in ("models", "spectra", "status")}
    ref = refs["models"]
    ref32 = np.concatenate([po.Restatement(po.LineSetup(l, LINE.lambda0, c["cuantic"], c["psf"], 9), "f32")
                            .invert(obs[i:i + 1], c["guess"], fix=c["fix"], noise=NOISE32)["models"]
                            for i, l in enumerate(lam)])
    with zinv(c, pm.PREC_FP64, pm.SOLVE_EIGEN) as inv:
        r64 = inv.invert(obs, c["guess"], lam=lam)
    with zinv(c, pm.PREC_FP32) as inv:
        r32 = inv.invert(obs, c["guess"], lam=lam)
    fast = None
    if po.reference_available("f64_fast"):
        fast = {"models": np.concatenate([po.Reference(o.setup, "f64_fast").invert(
            obs[i:i + 1], c["guess"], fix=c["fix"], noise=NOISE64, want_spectra=False)["models"]
            for i, o in enumerate(oras)])}
    assert_plain_parity(r64, refs, params=tuple(i for i in range(11) if c["fix"][i]), fast=fast, min_converged=0.0)
    dB = np.abs(r32["models"][:, 1] - ref[:, 1])
    assert np.median(dB) < 1.0
    assert (dB < 5.0).mean() >= _fp32_bar(np.abs(ref32[:, 1] - ref[:, 1]))


def test_server_serves_multiplet_grids_together():
    """Two multiplet grids in one server (30 points at 25 mA, 15 points at 50 mA):
    a scan gives the same results alone and among scans of the other grid, bit
    for bit, and the FP32 batch entry point's within the stated tolerance."""
    c = zcase("z9")
    lam15 = c["lam"][::2]
    psf15 = pm.psf_gaussian(60.0, lam15)
    g0 = pm.Grid(lam=c["lam"], psf=c["psf"], guess=c["guess"], noise=NOISE64, fix=c["fix"], nterms=9)
    g1 = pm.Grid(lam=lam15, psf=psf15, guess=c["guess"], noise=NOISE64, fix=c["fix"], nterms=9)
    obs0 = _observed(c, 44)
    ora15 = po.Restatement(po.LineSetup(lam15, LINE.lambda0, c["cuantic"], psf15, 9), "f64")
    rng = np.random.default_rng(45)
    obs1 = np.array([ora15.synth(m, fix=c["fix"], rf=False)[0] for m in _models(c, 64, 46)[-64:]], dtype=np.float32)
    obs1 += rng.normal(0, 1e-3, obs1.shape).astype(np.float32)
    with pm.Server(LINE, [g0, g1], hbm_budget_bytes=1 << 28) as srv:
        alone = srv.wait(srv.submit(0, obs0))
        ids = [srv.submit(1, obs1), srv.submit(0, obs0), srv.submit(1, obs1)]
        res = [srv.wait(i) for i in ids]
    for k in ("models", "chisq", "iters", "status"):
        assert np.array_equal(res[1][k], alone[k]), k
        assert np.array_equal(res[2][k], res[0][k]), k
    for g, obs, r in ((g0, obs0, alone), (g1, obs1, res[0])):
        with pm.Inverter(LINE, g.lam, g.psf, noise=NOISE64, fix=c["fix"], nterms=9, precision=pm.PREC_FP32) as inv:
            b = inv.invert(obs, c["guess"])
        dB = np.abs(r["models"][:, 1] - b["models"][:, 1])
        assert np.median(dB) < 1.0 and (dB < 5.0).mean() >= 0.85


def test_single_grid_server_matches_the_batch_entry_point():
    """A server with one multiplet grid inverts with the batch entry point's
    kernel: the FP32 results of both within the stated tolerance."""
    c = zcase("z9")
    g = pm.Grid(lam=c["lam"], psf=c["psf"], guess=c["guess"], noise=NOISE64, fix=c["fix"], nterms=9)
    with pm.Server(LINE, [g], hbm_budget_bytes=1 << 28) as srv:
        r = srv.wait(srv.submit(0, np.ascontiguousarray(c["obs"])))
    with zinv(c, pm.PREC_FP32) as inv:
        b = inv.invert(c["obs"], c["guess"])
    dB = np.abs(r["models"][:, 1] - b["models"][:, 1])
    assert np.median(dB) < 1.0 and (dB < 5.0).mean() >= 0.85


def test_nine_component_line_matches_oracle():
    """Fe I 15652.857 (7D5.0-7K4.0: nine pi and nine sigma components per group)
    on 30 wavelengths with a 60 mA PSF: FP64 synthesis and response functions,
    and FP64 inversions, against the oracle."""
    lam0, q = 15652.857, (3.0, 2.0, 5.0, 3.0, 7.0, 4.0)
    lam = lam0 + np.linspace(-0.6, 0.6, 30)
    psf = pm.psf_gaussian(60.0, lam)
    line = pm.line_from_quantum(lam0, *q)
    assert (line._c.n_pi, line._c.n_sig) == (9, 9)
    fix = [1] * 9 + [0, 0]
    ora = po.Restatement(po.LineSetup(lam, lam0, np.array([1.0, *q]), psf, 9), "f64")
    rng = np.random.default_rng(91)
    n = 48
    m = np.zeros((n, 11))
    m[:, 0] = rng.uniform(1, 20, n)
    m[:, 1] = rng.uniform(0, 2000, n)
    m[:, 2] = rng.uniform(-3, 3, n)
    m[:, 3] = rng.uniform(0.05, 0.12, n)
    m[:, 4] = rng.uniform(0.01, 0.5, n)
    m[:, 5] = rng.uniform(0, 180, n)
    m[:, 6] = rng.uniform(0, 180, n)
    m[:, 7] = rng.uniform(0.1, 0.4, n)
    m[:, 8] = rng.uniform(0.4, 0.9, n)
    m[:, 10] = 1.0
    guess = np.array([8.0, 400.0, 0.0, 0.08, 0.1, 30.0, 30.0, 0.25, 0.75, 0.0, 1.0])
    with pm.Inverter(line, lam, psf, noise=NOISE64, fix=fix, nterms=9, precision=pm.PREC_FP64,
                     solver=pm.SOLVE_EIGEN) as inv:
        sp, rf = inv.synth(m, rf=True)
        for i in range(n):
            s_ref, rf_ref = ora.synth(m[i], fix=fix)
            assert np.abs(sp[i] - s_ref).max() < 1e-6
            scale = np.abs(rf_ref).max(axis=-1, keepdims=True) + 1e-30
            assert (np.abs(rf[i] - rf_ref) / scale).max() < 1e-5
        obs = np.ascontiguousarray(sp + rng.normal(0, 1e-3, sp.shape), dtype=np.float32)
        r = inv.invert(obs, guess)
    ref = ora.invert(obs, guess, fix=fix, noise=NOISE64)
    assert within_tolerance(r["models"], ref["models"]).mean() >= 0.85
