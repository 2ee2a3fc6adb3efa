"""GPU inversion (pm_invert_batch / pm_lm_mils) against the oracle.

The plain form (FP64, eigen-decomposition solve) is the correctness twin of the
reference's double build: for pixels where both converge, parameters must agree
within |dB| < 1 G, angles < 0.1 deg, v_los < 1 m/s and 1e-4 relative for the
others and best-fit profiles within 1e-6 I_c (gpu_common.assert_plain_parity);
chi^2 and iteration-count histograms are compared.  The FP32 form is
checked against the FP64 oracle with its own stated tolerance."""
import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from gpu_common import (LINE_6173, NOISE64, assert_plain_parity, case, inverter, oracle, reference_fast,
                        within_tolerance)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle_results():
    out = {}
    for cfg in (0, 1, 2):
        c = case(cfg)
        out[cfg] = oracle(c).invert(c["obs"], c["guess"], slight=c["slight"], fix=c["fix"], noise=NOISE64)
    return out


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_plain_fp64_matches_oracle(cfg, oracle_results):
    c = case(cfg)
    ref = oracle_results[cfg]
    with inverter(c, pm.PREC_FP64, pm.SOLVE_EIGEN) as inv:
        r = inv.invert(c["obs"], c["guess"], slight=c["slight"])
    fast = reference_fast(po.LineSetup(c["lam"], LINE_6173[0], np.array([1.0, *LINE_6173[1]]), c["psf"], c["nterms"]))
    fast_r = None if fast is None else fast.invert(c["obs"], c["guess"], slight=c["slight"], fix=c["fix"],
                                                   noise=NOISE64, want_spectra=False)
    ok = assert_plain_parity(r, ref, params=tuple(i for i in range(11) if c["fix"][i]), fast=fast_r,
                             min_converged=0.2)
    # chi^2 and iteration-count histograms
    assert np.allclose(np.sort(r["chisq"][ok]), np.sort(ref["chisq"][ok]), rtol=1e-3)
    assert abs(np.median(r["iters"]) - np.median(ref["iters"])) <= 2


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_cholesky_fp64_matches_eigen(cfg):
    c = case(cfg)
    with inverter(c, pm.PREC_FP64, pm.SOLVE_EIGEN) as a, inverter(c, pm.PREC_FP64, pm.SOLVE_CHOLESKY) as b:
        ra = a.invert(c["obs"], c["guess"], slight=c["slight"])
        rb = b.invert(c["obs"], c["guess"], slight=c["slight"])
    assert within_tolerance(rb["models"], ra["models"]).mean() >= 0.9


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_fp32_batched_against_fp64_oracle(cfg, oracle_results):
    c = case(cfg)
    ref = oracle_results[cfg]
    with inverter(c, pm.PREC_FP32) as inv:
        r = inv.invert(c["obs"], c["guess"], slight=c["slight"])
    # stated FP32 tolerance: |dB| < 5 G, angles < 0.5 deg, v < 5 m/s, 1e-3 relative (90% of pixels)
    dB = np.abs(r["models"][:, 1] - ref["models"][:, 1])
    assert np.median(dB) < 1.0
    assert (dB < 5.0).mean() >= 0.9
    assert np.isfinite(r["models"]).all() and np.isfinite(r["chisq"]).all()


def test_ghosts_nfree_and_empty():
    c = case(0)
    obs = c["obs"][:4].copy()
    obs[1] = -5.0                      # every point masked: nfree < 0 would be garbage; all ghosts
    obs[2, :, :] = -5.0
    obs[2, 0, :] = c["obs"][2, 0, :]   # only Stokes I kept: 30 points
    obs[2, 0, :21] = -5.0              # 9 points left = NTERMS -> nfree == 0
    with inverter(c, pm.PREC_FP64) as inv:
        r = inv.invert(obs, c["guess"])
        assert r["status"][2] == pm.PIX_NFREE and r["iters"][2] == -1
        assert r["status"][0] in (pm.PIX_CONVERGED, pm.PIX_LAMBDA, pm.PIX_MAXITER)
        e = inv.invert(np.zeros((0, 4, c["lam"].size), np.float32), c["guess"])
        assert e["models"].shape == (0, 11)
    ref = oracle(c).invert(obs, c["guess"], fix=c["fix"], noise=NOISE64)
    assert ref["iters"][2] == -1


def test_lm_mils_batch_of_one_equals_batch():
    c = case(1)
    with inverter(c, pm.PREC_FP64) as inv:
        r = inv.invert(c["obs"][:3], c["guess"])
        for i in range(3):
            rc, m, sp, chi, it = inv.lm_mils(c["obs"][i], c["guess"])
            assert rc == 1 and it == r["iters"][i]
            assert np.array_equal(m, r["models"][i]) and chi == r["chisq"][i]
            assert np.array_equal(sp, r["spectra"][i])


def test_device_path_equals_host_path_and_batch_independence():
    import torch

    c = case(2)
    with inverter(c, pm.PREC_FP32) as inv:
        host = inv.invert(c["obs"], c["guess"], slight=c["slight"])
        dev = inv.invert(torch.as_tensor(c["obs"], device="cuda"), c["guess"],
                         slight=torch.as_tensor(c["slight"], dtype=torch.float32, device="cuda"))
        assert np.array_equal(host["models"], dev["models"].cpu().numpy())
        # each pixel is independent: alone == in the batch, bit for bit
        for i in (0, 17, 47):
            one = inv.invert(c["obs"][i:i + 1], c["guess"], slight=c["slight"])
            assert np.array_equal(one["models"][0], host["models"][i])
            assert np.array_equal(one["spectra"][0], host["spectra"][i])


def test_stats_counters():
    c = case(1)
    with inverter(c, pm.PREC_FP32) as inv:
        r = inv.invert(c["obs"], c["guess"])
        s = inv.stats()
    assert s["pixels"] == c["obs"].shape[0]
    assert s["iterations"] == int(r["iters"].clip(min=0).sum())
    assert 0 < s["accepted"] <= s["iterations"]
    assert s["kernel_ms"] > 0 and s["total_ms"] >= s["kernel_ms"]
