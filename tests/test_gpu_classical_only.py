"""The classical-estimates-only mode on the GPU: pm_config.miter < 0, the
reference's NumberOfCycles < 0 (milos.c:399-520), estimacionesClasicas from the
initial model with forInitialUse = 0 and no LM.  Cubes of
tests/golden/ref_classical_only.npz (configurations 0, 1, 2 on 30 wavelengths,
49 and 112 wavelengths); the expected models are the oracle restatement's, which
equals the reference bit for bit on them (tests/test_oracle_pin.py).  The
estimates are FP64 in both precisions (the sums run in another order than the
reference's loop, hence a 1e-7 tolerance rather than equality).
"""
import os

import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from conftest import GOLDEN
from gpu_common import NOISE64

pytestmark = pytest.mark.gpu

CE = np.load(os.path.join(GOLDEN, "ref_classical_only.npz"))
QUANTUM = (2.0, 1.0, 1.0, 2.0, 2.0, 0.0)  # 5P1.0-5D0.0
FIX9 = [1] * 9 + [0, 0]


def ce_case(name):
    g = lambda k: CE[f"{name}_{k}"]
    return g("lam"), float(g("lambda0")), g("obs"), g("guess")


def oracle_models(lam, l0, obs, guess):
    ora = po.Restatement(po.LineSetup(lam, l0, np.array([1.0, *QUANTUM]), None, 9), "f64")
    return np.array([ora.classical(o, guess, initial_use=False) for o in obs])


@pytest.mark.parametrize("prec", [pm.PREC_FP64, pm.PREC_FP32])
@pytest.mark.parametrize("name", ["c0", "c1", "c2", "w49", "w112"])
def test_classical_only_matches_the_oracle(name, prec):
    lam, l0, obs, guess = ce_case(name)
    with pm.Inverter(pm.LineData(l0, QUANTUM), lam, None, noise=NOISE64, fix=FIX9, nterms=9, miter=-1,
                     precision=prec) as inv:
        r = inv.invert(obs, guess)
    ref = oracle_models(lam, l0, obs, guess)
    assert np.allclose(r["models"], ref, rtol=1e-7, atol=1e-7)
    assert not np.allclose(r["models"][:, 7], guess[7])  # S0 holds B_los
    assert np.all(r["iters"] == 0) and np.all(r["chisq"] == 0)
    assert np.all(r["status"] == 3)  # PM_PIX_CLASSICAL
    assert np.all(r["spectra"] == 0)


@pytest.mark.parametrize("name", ["c1", "w112"])
def test_classical_only_device_buffers_equal_host_buffers(name):
    import torch

    lam, l0, obs, guess = ce_case(name)
    big = np.tile(obs, (50, 1, 1))
    with pm.Inverter(pm.LineData(l0, QUANTUM), lam, None, noise=NOISE64, fix=FIX9, nterms=9, miter=-1) as inv:
        host = inv.invert(big, guess)
        dev = inv.invert(torch.from_numpy(big).cuda(), guess)
    for k in ("models", "iters", "chisq", "status"):
        assert np.array_equal(dev[k].cpu().numpy(), host[k]), k
    n = obs.shape[0]
    assert np.array_equal(host["models"].reshape(50, n, 11), np.broadcast_to(host["models"][:n], (50, n, 11)))


def test_the_server_takes_no_classical_only_grid():
    lam, l0, obs, guess = ce_case("c1")
    g = pm.Grid(lam=lam, guess=guess, noise=NOISE64, fix=FIX9, nterms=9, miter=-1)
    with pytest.raises(pm.PmError) as e:
        pm.Server(pm.LineData(l0, QUANTUM), [g], hbm_budget_bytes=1 << 28)
    assert e.value.code == -22  # PM_EINVAL
