"""Real-time directory mode on the GPU: cubes written into a directory are
ingested on the device, served as device-resident scans, and their models
written next to them; the results equal the batch entry point's."""
import os
import threading
import time

import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from pmilos_b200 import workloads
from pmilos_b200.watch import DirectoryStream

pytestmark = pytest.mark.gpu


def test_directory_stream_serves_new_cubes(tmp_path):
    w = workloads.config(1, npix=48 * 64)
    with pm.Inverter(w.line, w.lam, w.psf, noise=w.noise, fix=w.fix, precision=pm.PREC_FP64) as inv64:
        cubes = [workloads.synthesize(w, inv_fp64=inv64, rng=np.random.default_rng(s)) for s in range(3)]
    rows, cols = 48, 64
    grid = pm.Grid(lam=w.lam, psf=w.psf, guess=w.guess, noise=w.noise, fix=w.fix, nterms=9)

    def write(k):
        # the reference's default order (lambda, Stokes, rows, columns), pixel = col * rows + row
        data = cubes[k].reshape(cols, rows, 4, w.nl)
        raw = po.fits_bytes(np.ascontiguousarray(data), ["WAVE-GRI", "STOKES", "HPLN-TAN", "HPLT-TAN"])
        tmp = tmp_path / f".cube{k}.tmp"
        tmp.write_bytes(raw)
        os.rename(tmp, tmp_path / f"cube{k}.fits")

    write(0)
    with pm.Server(w.line, [grid],
                   hbm_budget_bytes=1 << 30) as srv:
        stream = DirectoryStream(srv, 0, str(tmp_path), poll_s=0.02, timeout_s=1.0)
        late = threading.Timer(0.3, lambda: (write(1), write(2)))
        late.start()
        outs = stream.run()
        late.join()
    assert [os.path.basename(o) for o in outs] == ["cube0_mod_gpu.fits", "cube1_mod_gpu.fits", "cube2_mod_gpu.fits"]
    with pm.Inverter(w.line, w.lam, w.psf, noise=w.noise, fix=w.fix, precision=pm.PREC_FP32) as inv:
        for k, out in enumerate(outs):
            raw = open(out, "rb").read()
            planes = np.frombuffer(raw[2880:2880 + 4 * 13 * rows * cols], dtype=">f4").reshape(13, -1)
            ref = inv.invert(cubes[k], w.guess)
            dB = np.abs(planes[1] - ref["models"][:, 1])
            assert np.median(dB) < 1.0 and (dB < 5.0).mean() >= 0.9
            assert np.array_equal(planes[11], ref["iters"].astype(np.float32)) or \
                abs(np.median(planes[11]) - np.median(ref["iters"])) <= 2


def test_directory_stream_serves_wide_grid_cubes(tmp_path):
    """Cubes of the 112-point configuration-4 grid: the server runs one launch of
    the wide kernel per cube, and the model planes written equal the batch entry
    point's models bit for bit (as float32, the file's type)."""
    rows, cols = 24, 32
    w = workloads.config(4, npix=rows * cols)
    with pm.Inverter(w.line, w.lam, w.psf, noise=w.noise, fix=w.fix, precision=pm.PREC_FP64) as inv64:
        cubes = [workloads.synthesize(w, inv_fp64=inv64, rng=np.random.default_rng(10 + s)) for s in range(2)]
    for k, cube in enumerate(cubes):
        data = cube.reshape(cols, rows, 4, w.nl)
        raw = po.fits_bytes(np.ascontiguousarray(data), ["WAVE-GRI", "STOKES", "HPLN-TAN", "HPLT-TAN"])
        (tmp_path / f"wide{k}.fits").write_bytes(raw)
    grid = pm.Grid(lam=w.lam, psf=w.psf, guess=w.guess, noise=w.noise, fix=w.fix, nterms=9)
    with pm.Server(w.line, [grid], hbm_budget_bytes=1 << 30) as srv:
        outs = DirectoryStream(srv, 0, str(tmp_path), poll_s=0.02, timeout_s=0.5).run()
        st = srv.stats()
    assert sorted(os.path.basename(o) for o in outs) == ["wide0_mod_gpu.fits", "wide1_mod_gpu.fits"]
    assert st["kernel_launches"] == 2
    with pm.Inverter(w.line, w.lam, w.psf, noise=w.noise, fix=w.fix, precision=pm.PREC_FP32) as inv:
        for out in outs:
            k = int(os.path.basename(out)[4])
            raw = open(out, "rb").read()
            planes = np.frombuffer(raw[2880:2880 + 4 * 13 * rows * cols], dtype=">f4").reshape(13, -1)
            ref = inv.invert(cubes[k], w.guess)
            assert np.array_equal(planes[:11], ref["models"].T.astype(np.float32))
            assert np.array_equal(planes[11], ref["iters"].astype(np.float32))
