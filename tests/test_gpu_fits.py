"""Cube ingest on the GPU (pm_fits_reorder) against the reference's reader and
the restatement (see tests/test_fits.py), bit for bit, and on a cube of the
large-cube configuration's spectral shape (112 wavelengths) in the reference's
default order and in a transposed order."""
import os

import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from conftest import GOLDEN
from test_fits import CASES, N, SIZE, _case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", range(N))
def test_reorder_on_device_matches_reference(k):
    order, ct, raw, data = _case(k)
    cube = pm.ingest_fits(raw).cpu().numpy()
    assert np.array_equal(cube, po.fits_ingest(data, ct))
    if po.fits_roles([SIZE[r] for r in order], ct) != (0, 1, 2, 3):
        assert np.array_equal(cube, CASES[f"f{k}_ref"])


@pytest.mark.parametrize("order", ["LSRC", "RCLS", "SRCL"])
def test_reorder_wide_cube(order, tmp_path):
    size = {"R": 256, "C": 192, "L": 112, "S": 4}
    dims = [size[r] for r in order]
    rng = np.random.default_rng(5)
    data = rng.normal(size=dims[::-1]).astype(np.float32)
    ct = [{"R": "HPLN-TAN", "C": "HPLT-TAN", "L": "WAVE-GRI", "S": "STOKES"}[r] for r in order]
    path = tmp_path / "cube.fits"
    path.write_bytes(po.fits_bytes(data, ct))
    cube = pm.ingest_fits(str(path)).cpu().numpy()
    assert np.array_equal(cube, po.fits_ingest(data, ct))


@pytest.mark.parametrize("k", range(4))
def test_four_dimensional_stray_light_matches_the_reference_reader(k):
    """A 4-D stray-light cube (readFitsStrayLightFile, utilsFits.c:936-1180) is
    ingested on the device like an observed cube: a profile per pixel."""
    from pmilos_b200.files import read_stray_light_fits

    aux = np.load(os.path.join(GOLDEN, "fits_aux_cases.npz"))
    got = read_stray_light_fits(aux[f"s4_{k}_bytes"].tobytes())
    assert got.is_cuda
    assert np.array_equal(got.cpu().numpy(), aux[f"s4_{k}_ref"])
