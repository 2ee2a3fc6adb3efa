"""The drop-in exercised from C: tests/c_dropin/dropin.c, compiled with gcc
against include/pmilos.h and linked to libpmilos_b200.so.

* CPU: the struct layouts the C compiler gives the header (sizeof, offsetof)
  equal the ctypes mirrors of the Python interface, field by field.
* GPU: the C program does what the patched milos.c does in place of its
  per-pixel loop (milos.c:958-1009): one allocation per pixel packed into one
  cube, one pm_invert_batch call; then pm_lm_mils on a few pixels as a host that
  keeps the loop would.  Its results equal the Python interface's on the same
  inputs bit for bit, and each pm_lm_mils call equals its pixel of the batch.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import pmilos_b200 as pm
from gpu_common import LINE_6173, case, inverter

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "c_dropin", "dropin.c")
LIBDIR = os.path.dirname(pm.LIB_PATH)


@pytest.fixture(scope="module")
def dropin(tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    pm.load_library()  # built by the test session's set-up
    exe = str(tmp_path_factory.mktemp("dropin") / "dropin")
    subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", LIBDIR, "-lpmilos_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def _ctypes_layout():
    out = {}
    for cname, cls in (("pm_model", pm._Model), ("pm_line", pm._Line), ("pm_config", pm._Config),
                       ("pm_stats", pm._Stats), ("pm_tuning", pm._Tuning), ("pm_fits_cube", pm._FitsCube),
                       ("pm_server_config", pm._ServerConfig), ("pm_scan_info", pm._ScanInfo),
                       ("pm_server_stats", pm._ServerStats)):
        out[f"sizeof {cname}"] = ctypes.sizeof(cls)
        for f, _ in cls._fields_:
            out[f"offsetof {cname}.{f.rstrip('_')}"] = getattr(cls, f).offset
    return out


def test_header_struct_layouts_match_the_ctypes_mirrors(dropin):
    text = subprocess.run([dropin, "layout"], check=True, capture_output=True, text=True).stdout
    c = {}
    for line in text.splitlines():
        key, val = line.rsplit(" ", 1)
        c[key] = int(val)
    py = _ctypes_layout()
    assert set(py) <= set(c), sorted(set(py) - set(c))
    mismatch = {k: (c[k], py[k]) for k in py if c[k] != py[k]}
    assert not mismatch, mismatch
    assert c["abi_version"] == pm.load_library().pm_abi_version()


def _write_case(path, c, precision, n_single):
    nl = c["lam"].size
    obs = np.ascontiguousarray(c["obs"], dtype=np.float32)
    with open(path, "wb") as f:
        np.array([nl, obs.shape[0], c["nterms"], precision, c["psf"] is not None, n_single], np.int32).tofile(f)
        np.array([LINE_6173[0], *LINE_6173[1]], np.float64).tofile(f)
        np.asarray(c["lam"], np.float64).tofile(f)
        if c["psf"] is not None:
            np.asarray(c["psf"], np.float64).tofile(f)
        np.asarray(c["fix"], np.int32).tofile(f)
        np.asarray(c["guess"], np.float64).tofile(f)
        obs.tofile(f)


def _read_out(path, npix, nl, n_single):
    raw = open(path, "rb").read()
    off = 0

    def take(dtype, n):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=n, offset=off)
        off += a.nbytes
        return a

    out = {"models": take(np.float64, npix * 11).reshape(npix, 11), "chisq": take(np.float32, npix),
           "iters": take(np.int32, npix), "spectra": take(np.float32, npix * 4 * nl).reshape(npix, 4, nl),
           "single": []}
    for _ in range(n_single):
        out["single"].append(dict(rc=int(take(np.int32, 1)[0]), model=take(np.float64, 11),
                                  spectra=take(np.float32, 4 * nl).reshape(4, nl), chisq=take(np.float32, 1)[0],
                                  iter=int(take(np.int32, 1)[0])))
    assert off == len(raw)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,precision", [(1, pm.PREC_FP32), (0, pm.PREC_FP64)])
def test_c_host_drop_in_equals_the_python_interface(dropin, tmp_path, cfg, precision):
    c = case(cfg)
    n_single = 3
    _write_case(tmp_path / "in.bin", c, precision, n_single)
    subprocess.run([dropin, "invert", str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], check=True, timeout=300)
    got = _read_out(tmp_path / "out.bin", c["obs"].shape[0], c["lam"].size, n_single)
    with inverter(c, precision) as inv:
        ref = inv.invert(c["obs"], c["guess"])
    for k in ("models", "chisq", "iters", "spectra"):
        assert np.array_equal(got[k], ref[k]), k
    for i, s in enumerate(got["single"]):
        assert s["rc"] == 1 and s["iter"] == got["iters"][i]
        assert np.array_equal(s["model"], got["models"][i])
        assert s["chisq"] == got["chisq"][i]
        assert np.array_equal(s["spectra"], got["spectra"][i])
