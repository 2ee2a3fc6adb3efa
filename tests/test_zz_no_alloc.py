"""pm_invert_batch_noalloc: the inversion for hosts that may not allocate GPU memory.

Such callers (device memory reserved up front by another component,
allocation-free real-time loops, memory-accounted services) hand the library
host arrays and get results back without any cudaMalloc: the library stages
through a static device array built into it.  These tests call that entry point
through the C ABI and check that it returns exactly what the regular entry point
(pm_invert_batch through a context) returns -- the same compiled kernel, so the
same bits -- twice in a row, so that state left in the shared static array by one
call cannot leak into the next; and, in a fresh process, that a call leaves the
device's free memory unchanged.  The file sorts last so that a run stopping at
the first failure has run every other test.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import pmilos_b200 as pm
from gpu_common import case, inverter

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _same(a, b):
    for k in ("models", "chisq", "iters", "spectra", "status"):
        assert np.array_equal(a[k], b[k]), k


def _regular(c, precision):
    """A context with the launch tuning the no-alloc entry uses (the contexts'
    default: lock-step blocks of 8 pixels)."""
    inv = inverter(c, precision)
    inv.tuning = {"variant": 2, "warps_per_block": 8}
    return inv


@pytest.mark.parametrize("cfg,precision", [(1, pm.PREC_FP32), (1, pm.PREC_FP64), (2, pm.PREC_FP32)])
def test_noalloc_matches_regular_entry_twice(cfg, precision):
    c = case(cfg)
    with _regular(c, precision) as inv:
        ref = inv.invert(c["obs"], c["guess"], slight=c["slight"])
        first = inv.invert_noalloc(c["obs"], c["guess"], slight=c["slight"])
        second = inv.invert_noalloc(c["obs"], c["guess"], slight=c["slight"])
    _same(first, ref)
    _same(second, ref)


def test_noalloc_per_pixel_stray_light_and_a_smaller_second_call():
    c = case(2)
    sl = np.ascontiguousarray(np.broadcast_to(c["slight"].astype(np.float32), (c["obs"].shape[0], 4, c["lam"].size)))
    with _regular(c, pm.PREC_FP32) as inv:
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


# Run in a fresh process: the first call loads the kernels (module loading may
# reserve device memory once); the free device memory is then read around two
# further calls, one of them at the pixel limit.
_PROBE = r"""
import json, sys
import numpy as np
sys.path[:0] = [sys.argv[1], sys.argv[2], sys.argv[3]]
import torch
import pmilos_b200 as pm
from gpu_common import case, inverter
c = case(1)
big = np.ascontiguousarray(np.resize(c["obs"], (pm.NOALLOC_MAX_PIXELS, 4, c["lam"].size)))
with inverter(c, pm.PREC_FP32) as inv:
    inv.invert_noalloc(c["obs"], c["guess"])
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    a = inv.invert_noalloc(big, c["guess"])
    b = inv.invert_noalloc(c["obs"], c["guess"])
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
print(json.dumps({"free0": free0, "free1": free1, "iters": int(a["iters"].sum() + b["iters"].sum())}))
"""


def test_noalloc_call_leaves_free_device_memory_unchanged():
    env = dict(os.environ)
    out = subprocess.run([sys.executable, "-c", _PROBE, os.path.join(ROOT, "p-milos_b200"), HERE,
                          os.path.join(ROOT, "oracle")], capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert r["iters"] > 0
    assert r["free1"] == r["free0"], f"free device memory changed by {r['free0'] - r['free1']} bytes"
