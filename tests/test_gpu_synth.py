"""GPU synthesis and response functions (pm_synth_batch) against the oracle."""
import numpy as np
import pytest

import pmilos_b200 as pm
from gpu_common import case, inverter, oracle

pytestmark = pytest.mark.gpu

# typical LM step of each RF row: eta0, B, vlos, dopp, a, gamma, azimuth, S0, S1, alpha
STEP = np.array([0.1, 10.0, 0.01, 1e-3, 1e-2, 1.0, 1.0, 1e-2, 1e-2, 1e-2])


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


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_fp64_synthesis_and_rf_match_oracle(cfg):
    c = case(cfg)
    models = _models(256, cfg, stray=cfg == 2)
    with inverter(c, pm.PREC_FP64) as inv:
        sp, rf = inv.synth(models, slight=c["slight"], rf=True)
    ora = oracle(c)
    for i in range(models.shape[0]):
        s_ref, rf_ref = ora.synth(models[i], c["slight"], fix=c["fix"])
        # profiles within 1e-6 I_c (the GPU returns float32)
        assert np.abs(sp[i] - s_ref).max() < 1e-6
        scale = np.abs(rf_ref).max(axis=-1, keepdims=True) + 1e-30
        assert (np.abs(rf[i] - rf_ref) / scale).max() < 1e-5


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_fp32_synthesis_close_to_fp64_oracle(cfg):
    """FP32 profiles within 2e-6 I_c of the FP64 oracle.  FP32 response functions
    within the largest of: twice the error of the reference's own float build
    (REAL = float; the oracle's f32 flavour is bit-identical to it), 1% of the
    row's maximum, or 1e-6 I_c over a typical LM step of that parameter.  The RFs
    lose digits to cancellation in me_der's chain rule (the reference's float build
    is off by up to 25% of a row's maximum here), and weak-field Q, U response
    functions (~B^2) amplify the FP32 Voigt's far-wing error."""
    c = case(cfg)
    models = _models(256, 10 + cfg, stray=cfg == 2)
    with inverter(c, pm.PREC_FP32) as inv:
        sp, rf = inv.synth(models, slight=c["slight"], rf=True)
    o64, o32 = oracle(c, "f64"), oracle(c, "f32")
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


def test_device_pointer_synthesis_equals_host():
    import torch

    c = case(1)
    models = _models(100, 5)
    with inverter(c, pm.PREC_FP32) as inv:
        a = inv.synth(models)
        b = inv.synth(torch.as_tensor(models, device="cuda")).cpu().numpy()
    assert np.array_equal(a, b)
