"""Grids wider than one warp (33..128 wavelengths: two or four warps per pixel).

The cases are the 112-point Fe I 6302 grid of the large-cube configuration (25 mA
PSF, nine free parameters) and the 49-point grid of the reference's known-answer
test (60 mA PSF, stray light, filling factor inverted), from
tests/golden/ref_cases_wide.npz.  Observed profiles: the fixture's 16 pixels plus
pixels synthesized here by the FP64 oracle with seeded noise, some with ghost
wavelengths in the first, a middle and the last warp of the pixel.
"""
import os

import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from conftest import GOLDEN
from gpu_common import NOISE64, assert_plain_parity, reference_fast, within_tolerance

pytestmark = pytest.mark.gpu

WIDE = np.load(os.path.join(GOLDEN, "ref_cases_wide.npz"))
CUANTIC = (2.0, 1.0, 1.0, 2.0, 2.0, 0.0)
STEP = np.array([0.1, 10.0, 0.01, 1e-3, 1e-2, 1.0, 1.0, 1e-2, 1e-2, 1e-2])


def wcase(name, psf=True):
    g = lambda k: WIDE[f"{name}_{k}"]
    return dict(lam=g("lam"), lambda0=float(g("lambda0")), psf=g("psf") if (psf and g("psf").size) else None,
                slight=g("slight") if g("slight").size else None, obs=g("obs"), guess=g("guess"),
                fix=list(g("fix")), nterms=int(g("nterms")), truth=g("truth"))


def winverter(c, precision, solver=pm.SOLVE_DEFAULT):
    return pm.Inverter(pm.LineData(c["lambda0"], CUANTIC), c["lam"], c["psf"], noise=NOISE64, fix=c["fix"],
                       nterms=c["nterms"], precision=precision, solver=solver)


def woracle(c, flav="f64"):
    return po.Restatement(po.LineSetup(c["lam"], c["lambda0"], np.array([1.0, *CUANTIC]), c["psf"], c["nterms"]),
                          flav)


def _models(n, seed, stray=False):
    rng = np.random.default_rng(seed)
    m = np.zeros((n, 11))
    m[:, 0] = rng.uniform(1, 30, n)
    m[:, 1] = rng.uniform(0, 4000, n)
    m[:, 2] = rng.uniform(-5, 5, n)
    m[:, 3] = rng.uniform(0.015, 0.08, n)
    m[:, 4] = rng.uniform(0.005, 1.0, n)
    m[:, 5] = rng.uniform(0, 180, n)
    m[:, 6] = rng.uniform(0, 180, n)
    m[:, 7] = rng.uniform(0.05, 0.5, n)
    m[:, 8] = rng.uniform(0.3, 1.0, n)
    m[:, 10] = rng.uniform(0.6, 1.0, n) if stray else 1.0
    return m


def observed(c, n_extra, seed):
    """Fixture pixels + n_extra oracle-synthesized noisy pixels, with ghosts."""
    rng = np.random.default_rng(seed)
    truth = _models(n_extra, seed, stray=c["slight"] is not None)
    truth[:, 2] = rng.uniform(-3, 3, n_extra)
    truth[:, 3] = rng.uniform(0.02, 0.05, n_extra)
    truth[:, 4] = rng.uniform(0.01, 0.5, n_extra)
    ora = woracle(c)
    extra = np.array([ora.synth(m, c["slight"], fix=c["fix"], rf=False)[0] for m in truth], dtype=np.float32)
    extra += rng.normal(0, 1e-3, extra.shape).astype(np.float32)
    obs = np.concatenate([c["obs"], extra]).astype(np.float32)
    nl = c["lam"].size
    obs[2, :, 0] = -2.0               # leading ghost (first warp)
    obs[3, :, nl - 1] = -2.0          # trailing ghost (last warp)
    obs[4, 1, 40] = -1.5              # interior ghost in the second warp
    obs[5, :, :2] = -3.0              # two leading ghosts
    return np.ascontiguousarray(obs)


CASES = {}


def _case_results(name):
    if name not in CASES:
        c = wcase(name)
        obs = observed(c, 112, 7 if name == "w112" else 8)
        ref = woracle(c).invert(obs, c["guess"], slight=c["slight"], fix=c["fix"], noise=NOISE64)
        CASES[name] = (c, obs, ref)
    return CASES[name]


def test_kat_synthesis_on_two_warps():
    """The reference's known-answer synthesis (49 wavelengths, stray light)."""
    k = np.load(os.path.join(GOLDEN, "kat_synthesis.npz"))
    line = pm.LineData(float(k["lambda0"]), tuple(k["cuantic"][1:]))
    for prec, tol in ((pm.PREC_FP64, 1e-6), (pm.PREC_FP32, 3e-6)):
        with pm.Inverter(line, k["lam"], None, noise=NOISE64, fix=[1] * 9 + [0, 1], nterms=int(k["nterms"]),
                         precision=prec) as inv:
            sp = inv.synth(k["model"][None, :], slight=k["slight"].astype(np.float32))
        assert np.abs(sp[0] - k["expected"]).max() < tol, prec


@pytest.mark.parametrize("name,psf", [("w112", True), ("w112", False), ("w49", True), ("w49", False)])
def test_fp64_wide_synthesis_and_rf_match_oracle(name, psf):
    c = wcase(name, psf)
    models = _models(96, 3, stray=c["slight"] is not None)
    with winverter(c, pm.PREC_FP64) as inv:
        sp, rf = inv.synth(models, slight=c["slight"], rf=True)
    ora = woracle(c)
    for i in range(models.shape[0]):
        s_ref, rf_ref = ora.synth(models[i], c["slight"], fix=c["fix"])
        assert np.abs(sp[i] - s_ref).max() < 1e-6
        scale = np.abs(rf_ref).max(axis=-1, keepdims=True) + 1e-30
        assert (np.abs(rf[i] - rf_ref) / scale).max() < 1e-5


@pytest.mark.parametrize("name", ["w112", "w49"])
def test_fp32_wide_synthesis_close_to_fp64_oracle(name):
    """The FP32 criterion of the one-warp grids (see test_gpu_synth)."""
    c = wcase(name)
    models = _models(96, 4, stray=c["slight"] is not None)
    with winverter(c, pm.PREC_FP32) as inv:
        sp, rf = inv.synth(models, slight=c["slight"], rf=True)
    o64, o32 = woracle(c, "f64"), woracle(c, "f32")
    worst, rel = 0.0, []
    for i in range(models.shape[0]):
        s_ref, rf_ref = o64.synth(models[i], c["slight"], fix=c["fix"])
        _, rf_r32 = o32.synth(models[i], c["slight"], fix=c["fix"])
        worst = max(worst, np.abs(sp[i] - s_ref).max())
        rowmax = np.abs(rf_ref).max(axis=-1)
        e_gpu = np.abs(rf[i] - rf_ref).max(axis=-1)
        e_r32 = np.abs(rf_r32 - rf_ref).max(axis=-1)
        floor = 1e-6 / STEP[: rf_ref.shape[1]][None, :]
        assert np.all(e_gpu <= np.maximum(np.maximum(2.0 * e_r32, 1e-2 * rowmax), floor))
        rel.append(np.median(e_gpu / (rowmax + 1e-30)))
    assert worst < 2e-6
    assert np.median(rel) < 1e-4


@pytest.mark.parametrize("name", ["w112", "w49"])
def test_plain_fp64_wide_matches_oracle(name):
    c, obs, ref = _case_results(name)
    with winverter(c, pm.PREC_FP64, pm.SOLVE_EIGEN) as inv:
        r = inv.invert(obs, c["guess"], slight=c["slight"])
    fast = reference_fast(po.LineSetup(c["lam"], c["lambda0"], np.array([1.0, *CUANTIC]), c["psf"], c["nterms"]))
    fast_r = None if fast is None else fast.invert(obs, c["guess"], slight=c["slight"], fix=c["fix"],
                                                   noise=NOISE64, want_spectra=False)
    ok = assert_plain_parity(r, ref, params=tuple(i for i in range(11) if c["fix"][i]), fast=fast_r,
                             min_converged=0.2)
    assert ok[:6].all()  # the ghost pixels
    assert np.allclose(np.sort(r["chisq"][ok]), np.sort(ref["chisq"][ok]), rtol=1e-3)
    assert abs(np.median(r["iters"]) - np.median(ref["iters"])) <= 2


@pytest.mark.parametrize("name", ["w112", "w49"])
def test_cholesky_fp64_wide_matches_eigen(name):
    c, obs, _ = _case_results(name)
    with winverter(c, pm.PREC_FP64, pm.SOLVE_EIGEN) as a, winverter(c, pm.PREC_FP64, pm.SOLVE_CHOLESKY) as b:
        ra = a.invert(obs, c["guess"], slight=c["slight"])
        rb = b.invert(obs, c["guess"], slight=c["slight"])
    assert within_tolerance(rb["models"], ra["models"]).mean() >= 0.9


@pytest.mark.parametrize("name", ["w112", "w49"])
def test_fp32_wide_against_fp64_oracle(name):
    c, obs, ref = _case_results(name)
    with winverter(c, pm.PREC_FP32) as inv:
        r = inv.invert(obs, c["guess"], slight=c["slight"])
    # stated FP32 tolerance: |dB| < 5 G for 90% of pixels, median below 1 G
    dB = np.abs(r["models"][:, 1] - ref["models"][:, 1])
    assert np.median(dB) < 1.0
    assert (dB < 5.0).mean() >= 0.9
    assert np.all(r["status"] >= 0)


def test_wide_grid_classical_estimates_match_oracle():
    """miter = 0 runs one LM step (lm_mils' loop is a do-while) from the classical
    estimates: the cross-warp ghost trimming and sums feed it directly."""
    c, obs, _ = _case_results("w112")
    ref = woracle(c).invert(obs, c["guess"], slight=c["slight"], fix=c["fix"], noise=NOISE64, miter=0)
    with pm.Inverter(pm.LineData(c["lambda0"], CUANTIC), c["lam"], c["psf"], noise=NOISE64, fix=c["fix"],
                     nterms=c["nterms"], precision=pm.PREC_FP64, miter=0) as inv:
        r = inv.invert(obs, c["guess"])
    assert np.allclose(r["models"], ref["models"], rtol=1e-6, atol=1e-6)


def test_host_buffers_in_many_chunks_equal_one_call(monkeypatch):
    """Host-buffer calls on wide grids run through two device buffer sets, the
    next chunk's copy overlapping this chunk's inversion: a 1 MB device budget
    splits 600 pixels into chunks; results equal the single-chunk call and the
    device-buffer call bit for bit, statistics add up."""
    import torch

    c, obs, _ = _case_results("w112")
    big = np.ascontiguousarray(np.tile(obs, (5, 1, 1))[:600])
    with winverter(c, pm.PREC_FP32) as inv:
        one = inv.invert(big, c["guess"])
        dev = inv.invert(torch.as_tensor(big, device="cuda"), c["guess"])
    monkeypatch.setenv("PMILOS_RESIDENT_MB", "1")
    with winverter(c, pm.PREC_FP32) as inv:
        many = inv.invert(big, c["guess"])
        st = inv.stats()
    for k in ("models", "chisq", "iters", "spectra", "status"):
        assert np.array_equal(many[k], one[k]), k
        assert np.array_equal(dev[k].cpu().numpy(), one[k]), k
    assert st["pixels"] == 600 and st["iterations"] == int(np.maximum(many["iters"], 0).sum())
