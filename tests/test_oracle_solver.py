"""The oracle's eigen-solver (stand-in for GSL gsl_eigen_symmv) validated by
properties, since no reference test pins the solve: the pseudo-inverse step
delta = V diag(1/w) V^T beta must match an independent pseudo-inverse with the
same absolute 1e-12 eigenvalue cut (mil_svd, milosUtils.c:237-271)."""
import numpy as np
import pytest

import pyoracle as po


def _ctx():
    lam = 6173.3354 + np.arange(30) * 0.025
    return po.Restatement(po.LineSetup(lam, 6173.3354, np.array([1.0, 2, 1, 1, 2, 2, 0]), None, 9), "f64")


@pytest.mark.parametrize("K", [9, 10])
def test_pseudo_inverse_matches_numpy(K):
    o = _ctx()
    rng = np.random.default_rng(K)
    for trial in range(50):
        # moderately conditioned: agreement with an independent pseudo-inverse
        J = rng.normal(size=(40, K)) * np.logspace(-1, 1, K)
        A = J.T @ J * (1 + 0.1 * np.eye(K))
        b = rng.normal(size=K)
        d = o.svd_solve(A, b)
        w, V = np.linalg.eigh(A)
        inv = np.where(np.abs(w) > 1e-12, 1.0 / w, 0.0)
        ref = V @ (inv * (V.T @ b))
        assert np.allclose(d, ref, rtol=1e-10, atol=1e-13 * np.abs(ref).max())
        # LM-like scaling (column norms spanning 7 decades): backward stability
        J = rng.normal(size=(40, K)) * np.logspace(-3, 4, K)
        A = J.T @ J * (1 + 0.1 * np.eye(K))
        d = o.svd_solve(A, b)
        assert np.linalg.norm(A @ d - b) <= 1e-12 * np.linalg.norm(A, 2) * np.linalg.norm(d) + 1e-12 * np.linalg.norm(b)


def test_zero_rows_give_zero_step():
    o = _ctx()
    rng = np.random.default_rng(3)
    J = rng.normal(size=(40, 9))
    J[:, 4] = 0.0
    A = J.T @ J
    b = J.T @ rng.normal(size=40)
    d = o.svd_solve(A, b)
    assert d[4] == 0.0
    keep = [i for i in range(9) if i != 4]
    ref = np.linalg.solve(A[np.ix_(keep, keep)], b[keep])
    assert np.allclose(d[keep], ref, rtol=1e-9)
