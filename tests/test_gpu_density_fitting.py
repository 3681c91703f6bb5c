"""Density-fitted J from the packed device output equals the same contraction
of the dense reference-layout tensors (drop-in three_center and two_center),
whole and computed window by window."""

import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

syn = importlib.import_module("electron-integral-playground_b200.synthetic")
pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
mi = importlib.import_module("electron-integral-playground_b200.molecular_integral")
df = importlib.import_module("electron-integral-playground_b200.density_fitting")


def test_metric_matrix_matches_two_center():
    import torch

    m = syn.attach_synthetic_basis(syn.organic_molecule(5, seed=40), aux_l_max=4, seed=2)
    ad = pu.form_auxiliary_pair_data(m)
    M = df.metric_matrix(torch, m, ad).cpu().numpy()
    want = mi.two_center(ad, m)
    tol = np.maximum(1e-12, 1e-13 * np.abs(want))
    assert np.all(np.abs(M - want) <= tol)


@pytest.mark.parametrize("window_bytes", [None, 2e6])
def test_density_fitted_j_matches_dense(window_bytes):
    """gamma and J against the dense contraction with the same fitting
    coefficients (the metric's conditioning would otherwise amplify rounding
    differences), and c against the Cholesky solve's residual."""
    m = syn.attach_synthetic_basis(syn.organic_molecule(7, seed=41), aux_l_max=4, seed=2)
    pd, ad = pu.form_pair_data(m, 1e-14), pu.form_auxiliary_pair_data(m)
    rng = np.random.default_rng(5)
    C = rng.standard_normal((m.n_ao, 6))
    D = C @ C.T / m.n_ao
    J3 = mi.three_center(pd, ad, m)
    J, c, gamma = df.coulomb_matrix(m, pd, ad, D, window_bytes=window_bytes)
    J, c, gamma = J.cpu().numpy(), c.cpu().numpy(), gamma.cpu().numpy()
    gamma_ref = np.einsum("Pmn,mn->P", J3, D)
    np.testing.assert_allclose(gamma, gamma_ref, rtol=0, atol=1e-12 * max(1.0, np.max(np.abs(gamma_ref))))
    # the metric of this basis has condition number ~1e11: check the solve
    # against numpy on the same device metric at the accuracy that allows
    import torch

    M_dev = df.metric_matrix(torch, m, ad).cpu().numpy()
    c_np = np.linalg.solve(M_dev, gamma)
    assert np.max(np.abs(c - c_np)) <= 1e-4 * np.max(np.abs(c_np))
    J_ref = np.einsum("Pmn,P->mn", J3, c)
    np.testing.assert_allclose(J, J_ref, rtol=0, atol=1e-12 * max(1.0, np.max(np.abs(J_ref))))
    np.testing.assert_allclose(J, J.T, rtol=0, atol=1e-12 * max(1.0, np.max(np.abs(J_ref))))
