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


def test_batch_coulomb_kernels_match_dense():
    """The library's gamma / J kernels over a whole batch (three molecules,
    one launch each) against the dense contraction of the drop-in tensors,
    and the full J (Cholesky solve included) against the single-molecule path."""
    import torch

    bt = importlib.import_module("electron-integral-playground_b200.batch")
    mols = [syn.attach_synthetic_basis(syn.organic_molecule(n, seed=50 + n), aux_l_max=4, seed=3) for n in (3, 6, 9)]
    pds = [pu.form_pair_data(m, 1e-14) for m in mols]
    ads = [pu.form_auxiliary_pair_data(m) for m in mols]
    rng = np.random.default_rng(8)
    Ds = []
    for m in mols:
        C = rng.standard_normal((m.n_ao, 4))
        Ds.append(C @ C.T / m.n_ao)
    b = bt.ThreeCenterBatch(mols, pds, ads, precision="fp64")
    b.alloc_output()
    b.run()
    b.status()
    factors = [torch.linalg.cholesky(df.metric_matrix(torch, m, ad)) for m, ad in zip(mols, ads)]
    bc = df.BatchCoulomb(torch, b, factors)
    D = torch.as_tensor(np.concatenate([d.ravel() for d in Ds]), device="cuda")
    bc.run(D)
    b.sync()
    gamma = bc.gamma.cpu().numpy()
    c = bc.c.cpu().numpy()
    for k, (m, pd, ad, Dm) in enumerate(zip(mols, pds, ads, Ds)):
        J3 = mi.three_center(pd, ad, m)
        a0, a1 = int(bc.aux_off[k]), int(bc.aux_off[k + 1])
        g_ref = np.einsum("Pmn,mn->P", J3, Dm)
        np.testing.assert_allclose(gamma[a0:a1], g_ref, rtol=0, atol=1e-12 * max(1.0, np.abs(g_ref).max()))
        J_ref = np.einsum("Pmn,P->mn", J3, c[a0:a1])
        Jk = bc.molecule_J(k).cpu().numpy()
        np.testing.assert_allclose(Jk, J_ref, rtol=0, atol=1e-12 * max(1.0, np.abs(J_ref).max()))
        J1, c1, _ = df.coulomb_matrix(m, pd, ad, Dm)
        np.testing.assert_allclose(Jk, J1.cpu().numpy(), rtol=0, atol=1e-9 * max(1.0, np.abs(J_ref).max()))
    # solves through the inverted factors (two matrix-vector products) give the
    # same J as the triangular substitutions
    inv = df.BatchCoulomb(torch, b, factors, inverse_factors=True)
    inv.run(D)
    b.sync()
    Jt, Ji = bc.J.cpu().numpy(), inv.J.cpu().numpy()
    np.testing.assert_allclose(Ji, Jt, rtol=0, atol=1e-10 * max(1.0, np.abs(Jt).max()))
    b.close()
