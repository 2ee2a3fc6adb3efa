"""pm_invert_batch_noalloc: the inversion for hosts that may not allocate GPU memory.

Such callers (device memory reserved up front by another component,
allocation-free real-time loops, memory-accounted services) hand the library
host arrays and get results back without any cudaMalloc: the library stages
through a static device array built into it.  These tests call that entry point
through the C ABI and check that it returns what the regular entry point
(pm_invert_batch through a context) returns, twice in a row so that state left in
the shared static array by one call cannot leak into the next.  The file sorts
last so that a run stopping at the first failure has run every other test.
"""
import numpy as np
import pytest

import pmilos_b200 as pm
from gpu_common import case, inverter, within_tolerance

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert np.array_equal(a["iters"], b["iters"])
    assert np.all(within_tolerance(a["models"], b["models"]))
    assert np.allclose(a["chisq"], b["chisq"], rtol=1e-6, atol=0)
    assert np.abs(a["spectra"] - b["spectra"]).max() <= 1e-6
    assert np.array_equal(a["status"], b["status"])


@pytest.mark.parametrize("cfg,precision", [(1, pm.PREC_FP32), (1, pm.PREC_FP64), (2, pm.PREC_FP32)])
def test_noalloc_matches_regular_entry_twice(cfg, precision):
    c = case(cfg)
    with inverter(c, precision) as inv:
        ref = inv.invert(c["obs"], c["guess"], slight=c["slight"])
        first = inv.invert_noalloc(c["obs"], c["guess"], slight=c["slight"])
        second = inv.invert_noalloc(c["obs"], c["guess"], slight=c["slight"])
    _same(first, ref)
    _same(second, ref)


def test_noalloc_per_pixel_stray_light_and_a_smaller_second_call():
    c = case(2)
    sl = np.ascontiguousarray(np.broadcast_to(c["slight"].astype(np.float32), (c["obs"].shape[0], 4, c["lam"].size)))
    with inverter(c, pm.PREC_FP32) as inv:
        ref = inv.invert(c["obs"], c["guess"], slight=sl, slight_mode=pm.SLIGHT_PER_PIXEL)
        big = inv.invert_noalloc(c["obs"], c["guess"], slight=sl, slight_mode=pm.SLIGHT_PER_PIXEL)
        small = inv.invert_noalloc(c["obs"][:5], c["guess"], slight=sl[:5], slight_mode=pm.SLIGHT_PER_PIXEL)
    _same(big, ref)
    _same(small, {k: v[:5] for k, v in ref.items()})


def test_noalloc_rejects_more_pixels_than_the_static_scratch_holds():
    c = case(1)
    n = pm.NOALLOC_MAX_PIXELS + 1
    obs = np.zeros((n, 4, c["lam"].size), dtype=np.float32)
    with inverter(c, pm.PREC_FP32) as inv:
        with pytest.raises(pm.PmError) as e:
            inv.invert_noalloc(obs, c["guess"])
        assert e.value.code == -34 and "at most 4096 pixels" in str(e.value)
        # a call at the limit is accepted
        r = inv.invert_noalloc(np.repeat(c["obs"][:1], pm.NOALLOC_MAX_PIXELS, axis=0), c["guess"],
                               want_spectra=False)
    assert np.all(r["iters"] == r["iters"][0])
