"""Parity at the scale of the 100-water cluster (300 atoms in a 15 A cube,
2400 orbital and 43,200 auxiliary functions; its whole packed (mu nu|P) is
806 GB, so it only ever runs in auxiliary windows).  Slices of whole auxiliary
shells are checked against the reference library, through the drop-in entry
point and through a window of the resident batch."""

import importlib
import types

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

syn = importlib.import_module("electron-integral-playground_b200.synthetic")
pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
mi = importlib.import_module("electron-integral-playground_b200.molecular_integral")
bt = importlib.import_module("electron-integral-playground_b200.batch")
sv = importlib.import_module("electron-integral-playground_b200.serving")


@pytest.fixture(scope="module")
def water100():
    m = syn.water100_cluster(0)
    return m, pu.form_pair_data(m, 1e-14), pu.form_auxiliary_pair_data(m)


def _slices_by_l(ad, n_aux):
    """The first slice (at most 9 functions of whole shells) holding each
    auxiliary angular momentum."""
    picked = {}
    for lo, hi, sub in sv.aux_slices(ad, n_aux, 9):
        for l in sub:
            picked.setdefault(l, (lo, hi, sub))
    return [picked[l] for l in sorted(picked)]


def _window_dense(b, pd, ad, lo, hi, n_ao, w):
    """Expand a window's packed blocks to the dense layout of functions [lo, hi)."""
    J = np.zeros((hi - lo, n_ao, n_ao))
    for (li, lj), p in pd.items():
        pairs = np.unique(np.stack([np.asarray(p.i_ao_start), np.asarray(p.j_ao_start)], 1), axis=0)
        for lk, a in ad.items():
            blk = b.window_block(0, li, lj, lk)
            if blk is None or blk[1] == 0 or blk[2] == 0:
                continue
            off, nsp, nax = blk
            ni, nj, nk = 2 * li + 1, 2 * lj + 1, 2 * lk + 1
            arr = w[off:off + nsp * ni * nj * nk * nax].reshape(nsp, ni, nj, nk, nax)
            st = np.unique(np.asarray(a.i_ao_start))
            aux0 = st[(st >= lo) & (st < hi)] - lo
            assert pairs.shape[0] == nsp and aux0.shape[0] == nax
            I = pairs[:, 0][:, None, None, None, None] + np.arange(ni)[None, :, None, None, None]
            Jc = pairs[:, 1][:, None, None, None, None] + np.arange(nj)[None, None, :, None, None]
            K = aux0[None, None, None, None, :] + np.arange(nk)[None, None, None, :, None]
            I, Jc, K = np.broadcast_arrays(I, Jc, K)
            J[K, I, Jc] = arr
            off_diag = np.broadcast_to((pairs[:, 0] != pairs[:, 1])[:, None, None, None, None], arr.shape)
            J[K[off_diag], Jc[off_diag], I[off_diag]] = arr[off_diag]
    return J


def test_water100_aux_slices_against_reference(water100):
    import torch

    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference library not built")
    m, pd, ad = water100
    cases = _slices_by_l(ad, m.n_aux)
    assert {l for _, _, sub in cases for l in sub} >= {0, 1, 2, 3}
    b = bt.ThreeCenterBatch([m], [pd], [ad], precision="fp64")
    try:
        for lo, hi, sub in cases:
            proxy = types.SimpleNamespace(n_ao=m.n_ao, n_aux=hi - lo, spherical_basis=m.spherical_basis)
            want = oracle.drive_three_center(ref, pd, sub, proxy)
            got = mi.three_center(pd, sub, proxy)
            np.testing.assert_allclose(got, want, rtol=0, atol=1e-12, err_msg=f"drop-in [{lo}, {hi})")
            n = b.window([lo], [hi])
            out = torch.full((max(n, 1),), float("nan"), dtype=torch.float64, device="cuda")
            b.run_window(out.data_ptr())
            b.sync()
            b.status()
            dense = _window_dense(b, pd, ad, lo, hi, m.n_ao, out.cpu().numpy())
            np.testing.assert_allclose(dense, want, rtol=0, atol=1e-12, err_msg=f"window [{lo}, {hi})")
    finally:
        b.close()
