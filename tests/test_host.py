"""Host-side logic of the library (no GPU): the C ABI loads and exports every
symbol include/pmilos.h declares; the per-run precompute (Zeeman pattern, PSF
taps, grid) matches the reference; the file readers parse the reference's
formats."""
import os
import re

import numpy as np
import pytest

import pmilos_b200 as pm
import pyoracle as po
from conftest import GOLDEN, ROOT

PSF = np.load(os.path.join(GOLDEN, "ref_psf.npz"))


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "pmilos.h")).read()
    declared = set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(pm_\w+)\s*\(", hdr, re.M))
    assert declared == set(pm.EXPORTED_SYMBOLS)
    L = pm.load_library()
    for name in declared:
        assert hasattr(L, name), name
    assert L.pm_abi_version() == 2


def test_zeeman_triplet_matches_oracle():
    line = pm.line_from_quantum(6173.3354, 2, 1, 1, 2, 2, 0)
    c = line._c
    assert (c.n_pi, c.n_sig) == (1, 1)
    assert c.geff == pytest.approx(2.5, abs=1e-12)
    o = po.Restatement(po.LineSetup(np.linspace(6173.0, 6173.7, 30), 6173.3354, line.cuantic_dat(), None, 9),
                       "f64").cuantic()
    # N_PI, N_SIG, GL, GU, GEFF, FO, NUB, NUP, NUR, WEB, WEP, WER
    assert np.allclose(o, [1, 1, c.gl, c.gu, c.geff, 1.0, c.nub[0], c.nup[0], c.nur[0], c.web[0], c.wep[0],
                           c.wer[0]], rtol=0, atol=1e-12)


def test_zeeman_multiplet_normalised():
    line = pm.line_from_quantum(6301.5012, 2, 1, 2, 2, 2, 2)  # 5P2.0-5D2.0
    c = line._c
    assert (c.n_pi, c.n_sig) == (5, 4)
    assert sum(c.wep[:5]) == pytest.approx(1.0)
    assert sum(c.web[:4]) == pytest.approx(1.0) and sum(c.wer[:4]) == pytest.approx(1.0)


@pytest.mark.parametrize("name", ["c1", "c3a", "c3b", "c4", "kat"])
def test_psf_gaussian_matches_reference(name):
    g = pm.psf_gaussian(float(PSF[f"{name}_fwhm"]), PSF[f"{name}_lam"])
    assert np.allclose(g, PSF[f"{name}_fgauss"], rtol=1e-12, atol=1e-300)


@pytest.mark.parametrize("name", ["c1", "c3b", "c4", "kat"])
def test_psf_table_matches_reference(name):
    g = pm.psf_from_table(PSF[f"{name}_table_x"], PSF[f"{name}_table_y"], PSF[f"{name}_offs"])
    assert np.allclose(g, PSF[f"{name}_interp"], rtol=1e-12, atol=1e-300)


def test_psf_table_recentres_grid_without_zero_sample():
    # the 6-point grid has no zero offset: the reference shifts the table (milos.c:332-340)
    g = pm.psf_from_table(PSF["c3a_table_x"], PSF["c3a_table_y"], PSF["c3a_offs"])
    assert np.allclose(g, PSF["c3a_interp"], rtol=1e-12, atol=1e-300)
    assert abs(g.sum() - 1) < 1e-12


def test_psf_table_rejects_short_table():
    with pytest.raises(pm.PmError):
        pm.psf_from_table(np.arange(-100.0, 101.0), np.ones(201), np.arange(-350.0, 376.0, 25.0))


def test_grid_from_malla_is_cumulative():
    offs, lam = pm.grid_from_malla(-1204.0, 21.5, 1182.5, 6302.4936)
    assert lam.size == 112 and offs[56] == 0.0
    assert np.array_equal(lam, PSF["c4_lam"]) and np.array_equal(offs, PSF["c4_offs"])


def test_parse_lines_entries():
    idx, lam, q = pm.parse_lines_entry("1=FE 1   6173.3356    1.0   2.223 -2.880   5P 1.0- 5D 0.0  0.266  7.868e-15")
    assert (idx, lam, q) == (1, 6173.3356, (2.0, 1.0, 1.0, 2.0, 2.0, 0.0))
    idx, lam, q = pm.parse_lines_entry("3=FE 1   6302.4936    1.0   3.69    -0.97    5P 1.0- 5D 0.0  0.240599  2.9727e-14")
    assert (idx, lam) == (3, 6302.4936) and q == (2.0, 1.0, 1.0, 2.0, 2.0, 0.0)
    idx, lam, q = pm.parse_lines_entry("4=FE 1   5576.0990    2.5   3.43  -0.73    5F 1.0- 5D 0.0")
    assert q == (2.0, 3.0, 1.0, 2.0, 2.0, 0.0)


def test_file_readers(tmp_path):
    grid = tmp_path / "malla.grid"
    grid.write_text("IMPORTANT: header\n\nLine indices : Initial lambda Step Final lambda\n"
                    "-----------------------------------------------------------------------\n"
                    "1                       :        -350,            25,           375\n")
    assert pm.read_grid_file(str(grid)) == (1, -350.0, 25.0, 375.0)
    mod = tmp_path / "guess.mod"
    mod.write_text("eta_0 :8\nmagnetic field [G] :400\nLOS velocity [km/s] :0\nDoppler width [A] :0.03\n"
                   "damping :0.1\ngamma [deg] :30\nphi [deg] :30\nS_0 :0.25\nS_1 :0.75\nv_mac [km/s] :0\n"
                   "filling factor :1\n")
    assert np.array_equal(pm.read_model_file(str(mod)), [8, 400, 0, 0.03, 0.1, 30, 30, 0.25, 0.75, 0, 1])
    psf = tmp_path / "g.psf"
    psf.write_text("\t-1.0    0.25\n\t0.0    0.5\n\t1.0    0.25\n")
    x, y = pm.read_psf_file(str(psf))
    assert np.array_equal(x, [-1, 0, 1]) and np.array_equal(y, [0.25, 0.5, 0.25])


def test_trol_reader(tmp_path):
    names = ["Number of cycles (*):50", "Observed profiles (*):obs.fits", "Stray light file :",
             "PSF file :60", "Wavelength grid file (*):malla.grid", "Atomic parameters file (*):LINES",
             "Abundance file :", "Initial guess model 1 (*):guess.mod", "Initial guess model 2 :",
             "Weight for Stokes I :1", "Weight for Stokes Q :2", "Weight for Stokes U :2",
             "Weight for Stokes V :1", "AUTOMATIC SELECT. OF NODES? :",
             "Nodes for S_0 1 :1", "Nodes for S_1 1 :1", "Nodes for eta0 1 :1", "Nodes for magnetic field 1 :1",
             "Nodes for LOS velocity 1 :1", "Nodes for gamma 1 :1", "Nodes for phi 1 :0",
             "Nodes for lambda_doppler 1 :1", "Nodes for damping 1 :1", "Invert macroturbulence 1 :0"]
    names += ["x :"] * 10
    names += ["Invert filling factor? :", "Invert stray light factor? :1", "mu=cos (theta) :",
              "Estimated S/N for I :500", "Continuum contrast :", "Initial diagonal element :0.01",
              "Use FFT for convolutions :", "Diagonal element acceleration:1"]
    p = tmp_path / "a.mtrol"
    p.write_text("\n".join(n + " ! comment" for n in names) + "\n")
    c = pm.read_trol_file(str(p))
    assert c["cycles"] == 50 and c["weights"] == [1, 2, 2, 1]
    assert c["fix"] == [1, 1, 1, 1, 1, 1, 0, 1, 1, 0, 1]
    assert c["noise"] == pytest.approx(4e-6) and c["ilambda"] == 0.01 and c["logclambda"] == 1
    assert c["mu"] == 1.0 and c["psf_fwhm"] == 60.0


def _grid(nl, **kw):
    lam = 6173.3354 + np.linspace(-0.35, 0.35, nl)
    return pm.Grid(lam=lam, noise=1e-6, fix=[1] * 9 + [0, 0], nterms=9, **kw)


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the failure without a GPU")
def test_server_creation_checks_its_grids_then_needs_a_gpu():
    """pm_server_create validates the grids before it looks for a device: a
    classical-estimates-only grid (miter < 0) is refused, and a valid set -- grids
    of at most 32 wavelengths, wider ones, or both kinds together -- fails loudly
    without an sm_100 device (there is no CPU path)."""
    line = pm.LineData(6173.3354, (2.0, 1.0, 1.0, 2.0, 2.0, 0.0))
    with pytest.raises(pm.PmError) as e:
        pm.Server(line, [_grid(30, miter=-1)], hbm_budget_bytes=1 << 28)
    assert e.value.code == -22  # PM_EINVAL
    for grids in ([_grid(30), _grid(15)], [_grid(112), _grid(49)], [_grid(30), _grid(49)]):
        with pytest.raises(pm.PmError) as e:
            pm.Server(line, grids, hbm_budget_bytes=1 << 28)
        assert e.value.code == -19  # PM_ENODEV


LINES = np.load(os.path.join(GOLDEN, "ref_lines.npz"))


@pytest.mark.parametrize("idx", range(1, 10))
def test_zeeman_pattern_of_every_reference_line(idx):
    """pm_line_from_quantum against the reference's create_cuantic for every
    entry of its run/LINES: normal triplets and multiplets of up to nine
    components per group (Fe I 15652.857, 7D5.0-7K4.0)."""
    g = lambda k: LINES[f"l{idx}_{k}"]
    c = pm.line_from_quantum(float(g("lambda0")), *g("quantum"))._c
    ref = g("pattern")
    npi, nsig = int(ref[0]), int(ref[1])
    assert (c.n_pi, c.n_sig) == (npi, nsig)
    mine = [npi, nsig, c.gl, c.gu, c.geff, c.fo, *c.nub[:nsig], *c.nup[:npi], *c.nur[:nsig], *c.web[:nsig],
            *c.wep[:npi], *c.wer[:nsig]]
    assert np.allclose(mine, ref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("idx", range(1, 10))
def test_lines_entries_parse_like_the_reference(idx):
    """The LINES reader gives readFileCuanticLines' quantum numbers; entry 5's
    "7k", a letter the reference leaves undecoded (L unset), reads as K: L = 7."""
    text = str(LINES[f"l{idx}_text"])
    i, lam0, q = pm.files.parse_lines_entry(text)
    assert i == idx and lam0 == float(LINES[f"l{idx}_lambda0"])
    assert np.array_equal(np.array(q, dtype=np.float64), LINES[f"l{idx}_quantum"])
