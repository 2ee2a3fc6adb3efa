"""The real-time directory mode: the reference's file choice (alphabetical,
skipping outputs and directories and what was read before), CPU only."""
import os

import numpy as np

from pmilos_b200.watch import models_fits_bytes, new_cubes


def test_new_cubes_order_and_filter(tmp_path):
    for name in ["b.fits", "a.fits", "a_mod_gpu.fits", "x_stokes_1.fits", "c.fits", ".d.tmp"]:
        (tmp_path / name).write_bytes(b"")
    (tmp_path / "sub").mkdir()
    seen = {str(tmp_path / "c.fits")}
    got = new_cubes(str(tmp_path), seen)
    assert got == [str(tmp_path / "a.fits"), str(tmp_path / "b.fits")]


def test_models_fits_layout():
    rows, cols = 3, 5
    n = rows * cols
    models = np.arange(n * 11, dtype=np.float64).reshape(n, 11)
    iters = np.arange(n, dtype=np.int32)
    chisq = np.linspace(0, 1, n).astype(np.float32)
    raw = models_fits_bytes(models, iters, chisq, rows, cols)
    assert len(raw) % 2880 == 0
    data = np.frombuffer(raw[2880:2880 + 4 * 13 * n], dtype=">f4").reshape(13, n)
    assert np.array_equal(data[1], models[:, 1].astype(np.float32))
    assert np.array_equal(data[11], iters.astype(np.float32)) and np.array_equal(data[12], chisq)
    hdr = raw[:2880].decode("ascii")
    assert "NAXIS1  =                    3" in hdr and "NAXIS2  =                    5" in hdr
