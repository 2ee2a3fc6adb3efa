"""A Zeeman multiplet on the GPU: Fe I 6301.5012 (5P2.0-5D2.0; five pi and four
sigma components per group) on a 30-point grid, from
tests/golden/ref_cases_zeeman.npz (made by running the reference): z9 (60 mA PSF,
nine parameters), z10 (stray light, filling factor inverted).  The oracle equals
the reference bit for bit on these cases (tests/test_oracle_pin.py).
"""
import os

import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from conftest import GOLDEN
from gpu_common import NOISE64, within_tolerance

pytestmark = pytest.mark.gpu

ZEE = np.load(os.path.join(GOLDEN, "ref_cases_zeeman.npz"))
LINE = pm.LineData(6301.5012, (2.0, 1.0, 2.0, 2.0, 2.0, 2.0))
STEP = np.array([0.1, 10.0, 0.01, 1e-3, 1e-2, 1.0, 1.0, 1e-2, 1e-2, 1e-2, 1e-2])


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
    return np.concatenate([c["models"], m])


@pytest.mark.parametrize("name", ["z9", "z10"])
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


def test_fp32_synthesis_close_to_fp64_oracle():
    """The FP32 criterion of the other lines: profiles within 2e-6 of FP64, each
    response function no worse than the reference's own float build, or within
    1% of its row maximum, or within 1e-6 over a typical step."""
    c = zcase("z9")
    models = _models(c, 40, 22)
    with zinv(c, pm.PREC_FP32) as inv:
        sp, rf = inv.synth(models, rf=True)
    o64, o32 = zora(c, "f64"), zora(c, "f32")
    worst = 0.0
    for i in range(models.shape[0]):
        s_ref, rf_ref = o64.synth(models[i], fix=c["fix"])
        _, rf_r32 = o32.synth(models[i], fix=c["fix"])
        worst = max(worst, np.abs(sp[i] - s_ref).max())
        rowmax = np.abs(rf_ref).max(axis=-1)
        e_gpu = np.abs(rf[i] - rf_ref).max(axis=-1)
        e_r32 = np.abs(rf_r32 - rf_ref).max(axis=-1)
        floor = 1e-6 / STEP[: rf_ref.shape[1]][None, :]
        assert np.all(e_gpu <= np.maximum(np.maximum(2.0 * e_r32, 1e-2 * rowmax), floor))
    assert worst < 2e-6


@pytest.mark.parametrize("name", ["z9", "z10"])
def test_plain_fp64_inversion_matches_oracle(name):
    c = zcase(name)
    ref = zora(c).invert(c["obs"], c["guess"], slight=c["slight"], fix=c["fix"], noise=NOISE64)
    with zinv(c, pm.PREC_FP64, pm.SOLVE_EIGEN) as inv:
        r = inv.invert(c["obs"], c["guess"], slight=c["slight"])
    ok = within_tolerance(r["models"], ref["models"])
    assert ok.mean() >= 0.85, f"only {ok.mean():.2%} of pixels within tolerance"
    assert np.abs(r["spectra"][ok] - ref["spectra"][ok]).max() < 1e-5
    assert abs(np.median(r["iters"]) - np.median(ref["iters"])) <= 3


@pytest.mark.parametrize("name", ["z9", "z10"])
def test_fp32_inversion_against_fp64_oracle(name):
    c = zcase(name)
    ref = zora(c).invert(c["obs"], c["guess"], slight=c["slight"], fix=c["fix"], noise=NOISE64)
    with zinv(c, pm.PREC_FP32) as inv:
        r = inv.invert(c["obs"], c["guess"], slight=c["slight"])
    dB = np.abs(r["models"][:, 1] - ref["models"][:, 1])
    assert np.median(dB) < 1.0 and (dB < 5.0).mean() >= 0.85
    assert np.all(r["status"] >= 0)


def test_multiplet_limits():
    """Multiplets are compiled for one-warp grids without macroturbulence, and a
    server holds one alone (then with the batch entry point's kernel)."""
    c = zcase("z9")
    wide = np.linspace(6300.9, 6302.1, 49)
    with pytest.raises(pm.PmError) as e:
        pm.Inverter(LINE, wide, None, noise=NOISE64, fix=c["fix"], nterms=9)
    assert e.value.code == -95  # PM_ENOTSUP
    with pytest.raises(pm.PmError) as e:
        pm.Inverter(LINE, c["lam"], c["psf"], noise=NOISE64, fix=[1] * 10 + [0], nterms=10)
    assert e.value.code == -95
    g = pm.Grid(lam=c["lam"], psf=c["psf"], guess=c["guess"], noise=NOISE64, fix=c["fix"], nterms=9)
    with pytest.raises(pm.PmError) as e:
        pm.Server(LINE, [g, g], hbm_budget_bytes=1 << 28)
    assert e.value.code == -95
    with pm.Server(LINE, [g], hbm_budget_bytes=1 << 28) as srv:
        r = srv.wait(srv.submit(0, np.ascontiguousarray(c["obs"])))
    with zinv(c, pm.PREC_FP32) as inv:
        b = inv.invert(c["obs"], c["guess"])
    dB = np.abs(r["models"][:, 1] - b["models"][:, 1])
    assert np.median(dB) < 1.0 and (dB < 5.0).mean() >= 0.85
