"""Cube ingest on the CPU: the header parse of the C ABI and the restatement of
the reorder, against the reference's own FITS reader (readFitsSpectroImage run
over a CFITSIO read shim; tests/golden/fits_cases.npz, eight axis orders with and
without CTYPE cards).

The reference's special branch for the (rows, columns, wavelength, Stokes)
order (utilsFits.c:160, :228-241) indexes that order as if it were (wavelength,
Stokes, rows, columns); the ingest here applies the generic mapping
(utilsFits.c:242-336) to every order, so for that order only the restatement,
not the reference's output, is the expected result."""
import os

import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from conftest import GOLDEN

CASES = np.load(os.path.join(GOLDEN, "fits_cases.npz"))
N = len([k for k in CASES.files if k.endswith("_bytes")])
SIZE = {"R": 9, "C": 11, "L": 7, "S": 4}
ROLE = {"R": "HPLN-TAN", "C": "HPLT-TAN", "L": "WAVE-GRI", "S": "STOKES"}


def _case(k):
    order = str(CASES[f"f{k}_order"])
    ct = [ROLE[r] for r in order] if bool(CASES[f"f{k}_ctype"]) else None
    raw = CASES[f"f{k}_bytes"].tobytes()
    dims = [SIZE[r] for r in order]
    data = np.frombuffer(raw[2880:2880 + 4 * int(np.prod(dims))], dtype=">f4").reshape(dims[::-1])
    return order, ct, raw, data.astype(np.float32)


@pytest.mark.parametrize("k", range(N))
def test_header_parse_assigns_the_reference_roles(k):
    order, ct, raw, _ = _case(k)
    h = pm.fits_header(raw)
    dims = [SIZE[r] for r in order]
    assert h["naxes"] == dims and h["naxis"] == 4
    assert (h["axis_row"], h["axis_col"], h["axis_lambda"], h["axis_stokes"]) == po.fits_roles(dims, ct)
    assert h["from_ctype"] == (ct is not None)
    assert (h["nrows"], h["ncols"], h["nlambda"]) == (9, 11, 7) or ct is None
    assert h["data_offset"] == 2880 and h["data_bytes"] == 4 * int(np.prod(dims))


@pytest.mark.parametrize("k", range(N))
def test_restatement_matches_the_reference_reader(k):
    order, ct, raw, data = _case(k)
    mine = po.fits_ingest(data, ct)
    ref = CASES[f"f{k}_ref"]
    if po.fits_roles([SIZE[r] for r in order], ct) == (0, 1, 2, 3):
        assert not np.array_equal(mine, ref)  # the reference's special branch (see module docstring)
    else:
        assert np.array_equal(mine, ref)


def test_header_errors():
    data = np.zeros((4, 7, 3, 5), dtype=np.float32)
    ok = po.fits_bytes(data, None)
    with pytest.raises(pm.PmError):
        pm.fits_header(ok[:1000])                      # no END card
    bad = ok.replace(b"BITPIX  =                  -32", b"BITPIX  =                  -64")
    with pytest.raises(pm.PmError) as e:
        pm.fits_header(bad)
    assert e.value.code == -95
    three = po.fits_bytes(np.zeros((3, 7, 3, 5), dtype=np.float32), None)  # no 4-plane axis
    with pytest.raises(pm.PmError):
        pm.fits_header(three)


AUX = np.load(os.path.join(GOLDEN, "fits_aux_cases.npz"))


@pytest.mark.parametrize("k", range(4))
def test_two_dimensional_stray_light_matches_the_reference_reader(k):
    """readFitsStrayLightFile on (Stokes, lambda) and (lambda, Stokes) arrays:
    one profile [4][nlambda]."""
    from pmilos_b200.files import read_stray_light_fits

    got = read_stray_light_fits(AUX[f"s2_{k}_bytes"].tobytes())
    assert got.dtype == np.float32
    assert np.array_equal(got, AUX[f"s2_{k}_ref"])


@pytest.mark.parametrize("k", range(2))
def test_wavelength_file_matches_the_reference_reader(k):
    """readFitsLambdaToArray on a 2-D file (float64 and float32 pixels): the
    line index and the wavelengths."""
    from pmilos_b200.files import read_wavelength_fits

    idx, lam = read_wavelength_fits(AUX[f"l2_{k}_bytes"].tobytes())
    assert idx == int(AUX[f"l2_{k}_index"])
    assert np.array_equal(lam, AUX[f"l2_{k}_ref"])


def test_per_pixel_wavelength_file_round_trip():
    """The 4-D (per-pixel) wavelength file, which the reference documents but
    does not read: NAXIS1 = rows, NAXIS2 = columns, NAXIS3 = wavelength,
    NAXIS4 = 1, or axes named by CTYPE; pixel = column * rows + row."""
    from pmilos_b200.files import read_wavelength_fits

    rows, cols, nl = 5, 3, 7
    lam = 6173.0 + np.random.default_rng(3).uniform(0, 1, (cols * rows, nl))
    data = lam.reshape(cols, rows, nl).transpose(2, 0, 1)[None]  # numpy order (1, nl, cols, rows)
    raw = po.fits_bytes(data.astype(np.float32), None)
    idx, got = read_wavelength_fits(raw)
    assert idx is None and np.array_equal(got, lam.astype(np.float32).astype(np.float64))
    # the same grids with named axes in another order: (lambda, 1, rows, cols) as NAXIS1..4
    data2 = lam.reshape(cols, rows, nl)[:, :, None, :]  # numpy (cols, rows, 1, nl)
    raw2 = po.fits_bytes(data2.astype(np.float32), ["WAVE-GRI", "LINE", "HPLN-TAN", "HPLT-TAN"])
    _, got2 = read_wavelength_fits(raw2)
    assert np.array_equal(got2, got)
