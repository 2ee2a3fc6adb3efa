"""The serving loop (pm_server): continuous batching of scans on resident grids.

Grids: the served-stream configuration's three scans around Fe I 6173.3354 A --
6 points at +-172.5/+-103.5/+-34.5 mA, 15 points at 50 mA, 30 points at 25 mA --
with a 60 mA Gaussian PSF, nine free parameters, FP32.  Observed profiles are
synthesized by this library's FP64 path with seeded atmospheres (70% weak-field,
30% strong-field) and N(0, 1e-3) noise.
"""
import os

import numpy as np
import pytest

import pmilos_b200 as pm
from conftest import GOLDEN
from gpu_common import NOISE64, within_tolerance
from pmilos_b200 import workloads

pytestmark = pytest.mark.gpu

LINE = pm.LineData(workloads.FE6173, workloads.TRIPLET)


def grids():
    out = []
    for which in range(3):
        w = workloads.config(3, npix=1, grid=which)
        out.append(pm.Grid(lam=w.lam, psf=w.psf, guess=w.guess, noise=NOISE64, fix=w.fix, nterms=9))
    return out


def cube(which: int, npix: int, seed: int):
    w = workloads.config(3, npix=npix, grid=which)
    w.seed = seed
    return workloads.synthesize(w, rng=np.random.default_rng(seed))


@pytest.fixture(scope="module")
def cubes():
    return {(g, n, s): cube(g, n, s) for g, n, s in [(2, 3000, 1), (0, 20000, 2), (1, 9000, 3), (2, 5000, 4),
                                                      (0, 700, 5), (1, 64, 6)]}


def _eq(a, b):
    for k in ("models", "chisq", "iters", "status"):
        assert np.array_equal(a[k], b[k]), k


def test_scan_same_alone_and_in_the_mix(cubes):
    """A scan's results do not depend on what else is in flight: alone, and
    submitted among scans of all three grids, bit for bit (and so within the
    stated tolerance)."""
    A = cubes[(2, 3000, 1)]
    with pm.Server(LINE, grids(), hbm_budget_bytes=1 << 30, max_inflight=16) as srv:
        alone = srv.wait(srv.submit(2, A))
        ids = [srv.submit(0, cubes[(0, 20000, 2)]), srv.submit(1, cubes[(1, 9000, 3)]), srv.submit(2, A),
               srv.submit(2, cubes[(2, 5000, 4)]), srv.submit(0, cubes[(0, 700, 5)]), srv.submit(1, cubes[(1, 64, 6)])]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    mixed = res[2]
    _eq(alone, mixed)
    assert np.all(within_tolerance(mixed["models"], alone["models"]))
    # the mix overlapped: the repeated scan was admitted before the first scan of the mix finished
    assert res[2]["info"]["admit_ms"] < res[0]["info"]["done_ms"]
    assert st["scans_done"] == 7 and st["pixels_done"] == 3000 * 2 + 20000 + 9000 + 5000 + 700 + 64


def test_served_scans_match_the_batch_entry_point(cubes):
    """Every grid: the server's FP32 results against pm_invert_batch's FP32
    results on the same cube (the one-grid streamed kernel), within the stated
    FP32 tolerance; iteration statistics alike."""
    G = grids()
    with pm.Server(LINE, G, hbm_budget_bytes=1 << 30) as srv:
        for (g, n, s) in [(0, 700, 5), (1, 9000, 3), (2, 3000, 1)]:
            obs = cubes[(g, n, s)]
            r = srv.wait(srv.submit(g, obs))
            with pm.Inverter(LINE, G[g].lam, G[g].psf, noise=NOISE64, fix=G[g].fix, nterms=9,
                             precision=pm.PREC_FP32) as inv:
                b = inv.invert(obs, G[g].guess)
            dB = np.abs(r["models"][:, 1] - b["models"][:, 1])
            assert np.median(dB) < 1.0 and (dB < 5.0).mean() >= 0.9, g
            assert abs(np.median(r["iters"]) - np.median(b["iters"])) <= 2
            assert r["info"]["iterations"] == int(np.maximum(r["iters"], 0).sum())


def test_admission_respects_the_budget(cubes):
    """A budget that holds one scan at a time: every scan still completes, the
    arena never exceeds the budget, and a scan larger than the budget is refused."""
    A = cubes[(2, 3000, 1)]
    one_scan = 3000 * (4 * 30 * 4 + 88 + 12) + 4096
    with pm.Server(LINE, grids(), hbm_budget_bytes=max(one_scan, 1 << 20) + 1024, max_inflight=8) as srv:
        ids = [srv.submit(2, A) for _ in range(4)]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
        with pytest.raises(pm.PmError) as e:
            srv.submit(0, np.zeros((100000, 4, 6), dtype=np.float32))
        assert e.value.code == -34
    for r in res[1:]:
        _eq(r, res[0])
        assert r["info"]["admit_ms"] >= res[0]["info"]["admit_ms"]
    assert st["arena_peak_bytes"] <= max(one_scan, 1 << 20) + 1024
    # one scan at a time: each admission waited for the previous scan's results
    for a, b in zip(res, res[1:]):
        assert b["info"]["admit_ms"] >= a["info"]["done_ms"] - 1.0


def test_many_small_scans_share_a_kernel(cubes):
    """Continuous batching: scans submitted while the kernel runs join it, so
    there are far fewer kernel launches than scans."""
    small = cubes[(1, 64, 6)]
    big = cubes[(0, 20000, 2)]
    with pm.Server(LINE, grids(), hbm_budget_bytes=1 << 30, max_inflight=64, linger_ms=50.0) as srv:
        first = srv.submit(0, big)
        ids = [srv.submit(1, small) for _ in range(40)]
        res = [srv.wait(i) for i in ids]
        srv.wait(first)
        st = srv.stats()
    for r in res[1:]:
        _eq(r, res[0])
    assert st["kernel_launches"] <= 5, st
    # the persistent kernel computes the classical estimates itself: no pre-pass launches
    assert st["prepass_launches"] == 0, st
    assert st["latency_p99_ms"] >= st["latency_p50_ms"] > 0


def test_wait_timeout_and_unknown_id(cubes):
    with pm.Server(LINE, grids(), hbm_budget_bytes=1 << 30) as srv:
        sid = srv.submit(0, cubes[(0, 20000, 2)])
        with pytest.raises(TimeoutError):
            srv.wait(sid, timeout=0.0)
        r = srv.wait(sid)
        assert r["models"].shape == (20000, 11)
        with pytest.raises(pm.PmError):
            srv.wait(sid)
        with pytest.raises(pm.PmError):
            srv.submit(7, cubes[(0, 700, 5)])


# ---- grids of more than 32 wavelengths: one launch of the wide kernel per scan ----
WIDE_LINE = pm.LineData(6302.4936, (2.0, 1.0, 1.0, 2.0, 2.0, 0.0))
FIX9 = [1] * 9 + [0, 0]


def wide_grids():
    """The 112-point configuration-4 grid with its PSF (tests/golden/ref_cases_wide.npz)
    and every second point of it (56 points, 50 mA steps, a 25 mA Gaussian PSF)."""
    w = np.load(os.path.join(GOLDEN, "ref_cases_wide.npz"))
    lam, psf, guess = w["w112_lam"], w["w112_psf"], w["w112_guess"]
    lam56 = lam[::2].copy()
    return [pm.Grid(lam=lam, psf=psf, guess=guess, noise=NOISE64, fix=FIX9, nterms=9),
            pm.Grid(lam=lam56, psf=pm.psf_gaussian(25.0, lam56), guess=guess, noise=NOISE64, fix=FIX9, nterms=9)]


def wide_cube(g, npix, seed):
    """Profiles of seeded atmospheres synthesized in FP64 on the grid, N(0, 1e-3) noise."""
    rng = np.random.default_rng(seed)
    m = np.zeros((npix, 11))
    m[:, 0] = rng.uniform(1, 20, npix)
    m[:, 1] = rng.uniform(0, 3000, npix)
    m[:, 2] = rng.uniform(-3, 3, npix)
    m[:, 3] = rng.uniform(0.02, 0.05, npix)
    m[:, 4] = rng.uniform(0.01, 0.5, npix)
    m[:, 5] = rng.uniform(0, 180, npix)
    m[:, 6] = rng.uniform(0, 180, npix)
    m[:, 7] = rng.uniform(0.1, 0.4, npix)
    m[:, 8] = rng.uniform(0.4, 0.9, npix)
    m[:, 10] = 1.0
    with pm.Inverter(WIDE_LINE, g.lam, g.psf, noise=NOISE64, fix=FIX9, nterms=9, precision=pm.PREC_FP64) as inv:
        obs = inv.synth(m)
    return np.ascontiguousarray(obs + rng.normal(0, 1e-3, obs.shape), dtype=np.float32)


def test_wide_grid_scans_equal_the_batch_entry_point():
    """Each scan on a wide grid is one launch of the wide kernel after its copy-in:
    its results equal pm_invert_batch's on the same cube bit for bit, whatever
    else is queued, and every scan completes."""
    G = wide_grids()
    cubes = [wide_cube(G[0], 3000, 71), wide_cube(G[1], 2000, 72), wide_cube(G[0], 500, 73)]
    order = [(0, 0), (1, 1), (0, 2), (1, 1)]
    with pm.Server(WIDE_LINE, G, hbm_budget_bytes=1 << 30, max_inflight=8) as srv:
        ids = [srv.submit(g, cubes[c]) for g, c in order]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    for (g, c), r in zip(order, res):
        with pm.Inverter(WIDE_LINE, G[g].lam, G[g].psf, noise=NOISE64, fix=FIX9, nterms=9,
                         precision=pm.PREC_FP32) as inv:
            b = inv.invert(cubes[c], G[g].guess)
        _eq(r, b)
    assert st["scans_done"] == 4 and st["kernel_launches"] == 4
    assert st["pixels_done"] == 3000 + 2000 + 500 + 2000


def test_one_warp_and_wide_grids_in_one_server():
    """A server holding a 30-point grid (the persistent kernel) and the 112-point
    grid (one wide launch per scan): scans of both kinds, interleaved in the
    queue, each equal to pm_invert_batch's result on its grid bit for bit; the
    persistent kernel is closed before each wide scan and relaunched after it."""
    G = wide_grids()
    lam30 = G[0].lam[41:71].copy()
    g30 = pm.Grid(lam=lam30, psf=pm.psf_gaussian(25.0, lam30), guess=G[0].guess, noise=NOISE64, fix=FIX9, nterms=9)
    both = [g30, G[0]]
    cubes_ = {"a": wide_cube(g30, 4000, 81), "b": wide_cube(g30, 700, 82), "w": wide_cube(G[0], 1500, 83)}
    order = [(0, "a"), (1, "w"), (0, "b"), (1, "w"), (0, "a")]
    with pm.Server(WIDE_LINE, both, hbm_budget_bytes=1 << 30, max_inflight=8, linger_ms=20.0) as srv:
        ids = [srv.submit(g, cubes_[c]) for g, c in order]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    for (g, c), r in zip(order, res):
        with pm.Inverter(WIDE_LINE, both[g].lam, both[g].psf, noise=NOISE64, fix=FIX9, nterms=9,
                         precision=pm.PREC_FP32) as inv:
            b = inv.invert(cubes_[c], both[g].guess)
        _eq(r, b)
    assert st["scans_done"] == 5 and st["pixels_done"] == 4000 + 1500 + 700 + 1500 + 4000
    assert st["kernel_launches"] >= 4  # two wide launches, and the persistent kernel around them


# ---- stray light, as the reference's real-time loop applies its StrayLightFile ----
def test_shared_stray_light_scans_match_the_batch_entry_point():
    """A one-warp grid with a stray-light profile and the filling factor inverted
    (the 10-parameter configuration): the served FP32 results against
    pm_invert_batch's with the same profile, within the stated FP32 tolerance."""
    w = workloads.config(2, npix=3000)
    obs = workloads.synthesize(w, rng=np.random.default_rng(81))
    sl = np.asarray(w.slight, dtype=np.float32)
    g = pm.Grid(lam=w.lam, psf=w.psf, guess=w.guess, noise=NOISE64, fix=w.fix, nterms=w.nterms)
    line = pm.LineData(workloads.FE6173, workloads.TRIPLET)
    with pm.Server(line, [g], hbm_budget_bytes=1 << 28) as srv:
        srv.set_slight(0, sl)
        r = srv.wait(srv.submit(0, obs))
        with pytest.raises(pm.PmError) as e:  # only before the first submit
            srv.set_slight(0, None)
        assert e.value.code == -22
    with pm.Inverter(line, w.lam, w.psf, noise=NOISE64, fix=w.fix, nterms=w.nterms, precision=pm.PREC_FP32) as inv:
        b = inv.invert(obs, w.guess, slight=sl)
        unmixed = inv.invert(obs, w.guess)
    dB = np.abs(r["models"][:, 1] - b["models"][:, 1])
    assert np.median(dB) < 1.0 and (dB < 5.0).mean() >= 0.9
    da = np.abs(r["models"][:, 10] - b["models"][:, 10])
    assert np.median(da) < 1e-3
    # the profile is applied: without it the filling factors come out otherwise
    assert np.median(np.abs(unmixed["models"][:, 10] - b["models"][:, 10])) > 10 * max(np.median(da), 1e-6)


def test_per_pixel_stray_light_cube_on_a_wide_grid():
    """A [npix][4][nl] stray-light cube resident in the server (49 wavelengths,
    two warps per pixel): every scan's results equal pm_invert_batch's with the
    same cube bit for bit; a scan of another pixel count is refused."""
    w = np.load(os.path.join(GOLDEN, "ref_cases_wide.npz"))
    lam, psf, guess, fix = w["w49_lam"], w["w49_psf"], w["w49_guess"], list(w["w49_fix"])
    l0, nterms = float(w["w49_lambda0"]), int(w["w49_nterms"])
    line = pm.LineData(l0, (2.0, 1.0, 1.0, 2.0, 2.0, 0.0))
    rng = np.random.default_rng(82)
    npix = 1500
    cube = (w["w49_slight"][None].astype(np.float64) * rng.uniform(0.9, 1.1, (npix, 1, 1))).astype(np.float32)
    truth = np.repeat(guess[None], npix, axis=0)
    truth[:, 1] = rng.uniform(0, 3000, npix)
    truth[:, 2] = rng.uniform(-3, 3, npix)
    truth[:, 10] = rng.uniform(0.7, 1.0, npix)
    with pm.Inverter(line, lam, psf, noise=NOISE64, fix=fix, nterms=nterms, precision=pm.PREC_FP64) as inv:
        obs = inv.synth(truth, slight=cube)
    obs = np.ascontiguousarray(obs + rng.normal(0, 1e-3, obs.shape), dtype=np.float32)
    g = pm.Grid(lam=lam, psf=psf, guess=guess, noise=NOISE64, fix=fix, nterms=nterms)
    with pm.Server(line, [g], hbm_budget_bytes=1 << 28) as srv:
        srv.set_slight(0, cube)
        ids = [srv.submit(0, obs), srv.submit(0, obs)]
        res = [srv.wait(i) for i in ids]
        with pytest.raises(pm.PmError) as e:
            srv.submit(0, obs[:100])
        assert e.value.code == -22  # PM_EINVAL
    with pm.Inverter(line, lam, psf, noise=NOISE64, fix=fix, nterms=nterms, precision=pm.PREC_FP32) as inv:
        b = inv.invert(obs, guess, slight=cube)
    for r in res:
        _eq(r, b)
