"""Host-buffer pipelining, the launch tunings and graph replay.

Every one-warp inversion runs the streamed kernel.  Device-buffer calls publish
all pixels before one launch; host-buffer calls send the cube in up to
pm_tuning.staging_depth pieces of doubling size to one launch that inverts each
piece once the copy stream has published it.  Staging depth, pixels per block
and where the results are stored (device buffers copied back, or pinned host
arrays written by the kernel) do not change the compiled code, so results are
bit-identical across them and equal to the device-buffer call.  The two register budgets (pm_tuning.variant) are separately compiled
kernels whose floating-point contractions may differ in the last bits: between
them the stated FP32 tolerance applies.
"""
import numpy as np
import pytest
import torch

import pmilos_b200 as pm
from gpu_common import case, inverter

pytestmark = pytest.mark.gpu


def _device_reference(inv, c):
    obs_d = torch.as_tensor(c["obs"], device="cuda")
    sl = None if c["slight"] is None else torch.as_tensor(np.asarray(c["slight"], dtype=np.float32), device="cuda")
    r = inv.invert(obs_d, c["guess"], slight=sl)
    return {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in r.items()}


def _same(a, b):
    for k in ("models", "chisq", "iters", "spectra", "status"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("cfg", [0, 1, 2])
@pytest.mark.parametrize("precision", [pm.PREC_FP32, pm.PREC_FP64])
def test_every_tuning_gives_the_device_call_result(cfg, precision):
    c = case(cfg)
    with inverter(c, precision) as inv:
        refs = []
        for variant in ((0, 1) if precision == pm.PREC_FP32 else (0,)):
            inv.tuning = {"variant": variant, "staging_depth": 8, "warps_per_block": 4}
            ref = _device_reference(inv, c)
            refs.append(ref)
            for depth in (0, 1, 3, 64):
                for wpb in (1, 2, 4):
                    inv.tuning = {"variant": variant, "staging_depth": depth, "warps_per_block": wpb}
                    r = inv.invert(c["obs"], c["guess"], slight=c["slight"])
                    _same(r, ref)
        if precision == pm.PREC_FP32:
            # the lock-step kernel: the 128-register kernel's arithmetic, phase by phase
            for wpb in (4, 8, 16):
                inv.tuning = {"variant": 2, "staging_depth": 0, "warps_per_block": wpb}
                _same(_device_reference(inv, c), refs[1])
                inv.tuning = {"variant": 2, "staging_depth": 3, "warps_per_block": wpb}
                _same(inv.invert(c["obs"], c["guess"], slight=c["slight"]), refs[1])
    for other in refs[1:]:
        # the stated FP32 tolerance: |dB| < 5 G for 90% of pixels, median below 1 G
        dB = np.abs(other["models"][:, 1] - refs[0]["models"][:, 1])
        assert np.median(dB) < 1.0 and (dB < 5.0).mean() >= 0.9


def test_streamed_many_pieces_large_cube():
    """More pixels than pieces x 32, ragged last piece, per-pixel stray light."""
    c = case(2)
    reps = 70
    obs = np.ascontiguousarray(np.tile(c["obs"], (reps, 1, 1))[:3333])
    sl = np.ascontiguousarray(np.broadcast_to(np.asarray(c["slight"], dtype=np.float32), obs.shape))
    with inverter(c, pm.PREC_FP32) as inv:
        inv.tuning = {"staging_depth": 0}
        a = inv.invert(obs, c["guess"], slight=sl, slight_mode=pm.SLIGHT_PER_PIXEL)
        inv.tuning = {"staging_depth": 37}
        b = inv.invert(obs, c["guess"], slight=sl, slight_mode=pm.SLIGHT_PER_PIXEL)
        s = inv.stats()
    _same(a, b)
    assert s["pixels"] == obs.shape[0] and s["iterations"] == int(np.maximum(b["iters"], 0).sum())


def test_pinned_result_arrays_are_written_by_the_kernel():
    """Result arrays in pinned host memory (out=) receive the kernel's stores
    directly; the results equal those of pageable arrays and of the device call bit
    for bit, in one piece and in doubling pieces, with and without status and
    best-fit profiles, on both kernels."""
    c = case(1)
    n = 3333  # above the graph path's limit: the streamed host-buffer call
    obs = np.ascontiguousarray(np.tile(c["obs"], (n // c["obs"].shape[0] + 1, 1, 1))[:n])
    pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()
    with inverter(c, pm.PREC_FP32) as inv:
        for variant, wpb in ((1, 4), (2, 8)):
            inv.tuning = {"variant": variant, "warps_per_block": wpb, "staging_depth": 1}
            ref = _device_reference(inv, {**c, "obs": obs})
            for depth in (1, 5, 64):
                inv.tuning = {"variant": variant, "warps_per_block": wpb, "staging_depth": depth}
                out = {"models": pin((n, 11), torch.float64), "chisq": pin((n,), torch.float32),
                       "iters": pin((n,), torch.int32), "status": pin((n,), torch.int32),
                       "spectra": pin((n, 4, inv.nl), torch.float32)}
                for a in out.values():
                    a.fill(-7)
                r = inv.invert(obs, c["guess"], slight=c["slight"], out=out)
                assert all(r[k] is out[k] for k in out)
                _same(r, ref)
                # without status and profiles: only the arrays asked for are written
                out2 = {k: out[k] for k in ("models", "chisq", "iters")}
                for a in out2.values():
                    a.fill(-7)
                r2 = inv.invert(obs, c["guess"], slight=c["slight"], want_spectra=False, want_status=False, out=out2)
                for k in out2:
                    assert np.array_equal(r2[k], ref[k]), k
                # pageable arrays of the caller's own
                r3 = inv.invert(obs, c["guess"], slight=c["slight"], out={"models": np.empty((n, 11))})
                _same(r3, ref)
        with pytest.raises(ValueError):
            inv.invert(obs, c["guess"], out={"models": np.empty((n, 10))})


def test_unaligned_device_cube_gives_the_aligned_result():
    """The lock-step kernel reads a pixel's profiles with 16-byte loads when the
    cube starts on a 16-byte boundary and with 4-byte loads otherwise: a device
    cube one float into its buffer gives the aligned copy's results bit for bit."""
    c = case(1)
    obs = torch.as_tensor(c["obs"], device="cuda")
    buf = torch.empty(obs.numel() + 1, dtype=torch.float32, device="cuda")
    buf[1:].copy_(obs.reshape(-1))
    shifted = buf[1:].view(obs.shape)
    assert shifted.data_ptr() % 16 != 0 and obs.data_ptr() % 16 == 0
    with inverter(c, pm.PREC_FP32) as inv:
        for wpb in (8, 16):
            inv.tuning = {"variant": 2, "warps_per_block": wpb}
            a = inv.invert(obs, c["guess"])
            b = inv.invert(shifted, c["guess"])
            for k in ("models", "chisq", "iters", "spectra", "status"):
                assert torch.equal(a[k], b[k]), k


def test_autotune_picks_a_valid_tuning_and_keeps_results():
    c = case(1)
    with inverter(c, pm.PREC_FP32) as inv:
        t = inv.autotune(np.tile(c["obs"], (64, 1, 1)), c["guess"], reps=1)
        assert t == inv.tuning
        assert (t["variant"], t["warps_per_block"]) in {(v, w) for v in (0, 1) for w in (1, 2, 4)} | {(2, 8), (2, 16)}
        assert t["staging_depth"] in (0, 2, 4)
        # the chosen register budget's own device-buffer result
        _same(inv.invert(c["obs"], c["guess"]), _device_reference(inv, c))


def test_bad_tuning_is_rejected():
    c = case(1)
    with inverter(c, pm.PREC_FP32) as inv:
        for bad in ({"warps_per_block": 3}, {"staging_depth": 65}, {"variant": 3},
                    {"variant": 1, "warps_per_block": 8}, {"variant": 2, "warps_per_block": 2}):
            with pytest.raises(pm.PmError) as e:
                inv.tuning = bad
            assert e.value.code == -22


def test_small_calls_replay_a_captured_graph():
    """Host-buffer calls of <= PM_GRAPH_MAX_PIXELS pixels replay one CUDA graph per
    size: the first call captures, later ones replay; results equal the
    graph-free streamed call bit for bit, also after the parameters change."""
    c = case(2)
    with inverter(c, pm.PREC_FP32) as inv:
        inv.tuning = {"graphs": 0}
        ref = inv.invert(c["obs"], c["guess"], slight=c["slight"])
        assert inv.stats()["graph_replays"] == 0
        inv.tuning = {"graphs": 1}
        for _ in range(3):
            r = inv.invert(c["obs"], c["guess"], slight=c["slight"])
            assert inv.stats()["graph_replays"] == 1
            _same(r, ref)
        # another size, then a changed guess (a new parameter block) recapture
        r5 = inv.invert(c["obs"][:5], c["guess"], slight=c["slight"])
        _same({k: v for k, v in r5.items()}, {k: v[:5] for k, v in ref.items()})
        g2 = np.array(c["guess"], dtype=float)
        g2[1] = 900.0
        inv.tuning = {"graphs": 0}
        ref2 = inv.invert(c["obs"], g2, slight=c["slight"])
        inv.tuning = {"graphs": 1}
        _same(inv.invert(c["obs"], g2, slight=c["slight"]), ref2)
        # lm_mils, the batch of one, takes the graph path too
        rc, model, spectra, chi, it = inv.lm_mils(c["obs"][7], c["guess"], slight=c["slight"])
        assert np.array_equal(model, ref["models"][7]) and it == ref["iters"][7]


def test_stalled_queue_wait_is_bounded_and_reported():
    """A producer that never publishes cannot hang the device: the persistent
    kernel's wait gives up after its limit, says so in the queue's error word,
    and the context inverts normally afterwards."""
    c = case(1)
    with inverter(c, pm.PREC_FP32) as inv:
        err, ms = inv.selftest_stalled_queue(50.0)
        assert err == 1
        assert 40.0 <= ms < 2000.0
        ref = inv.invert(c["obs"], c["guess"])
        inv.tuning = {"graphs": 0, "staging_depth": 4}
        _same(inv.invert(c["obs"], c["guess"]), ref)
