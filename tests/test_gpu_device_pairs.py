"""Device-built pair tables against the vectorised front end (itself
bit-identical to the reference): same classes, same pairs in the same order,
values within 1e-12 relative (device exp/pow; the largest differences sit in
exp(-x) of large x, e.g. coefficients below 1e-100), and the integrals
computed from either agree."""

import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

syn = importlib.import_module("electron-integral-playground_b200.synthetic")
pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
dpairs = importlib.import_module("electron-integral-playground_b200.device_pairs")
mi = importlib.import_module("electron-integral-playground_b200.molecular_integral")


def _molecules():
    yield syn.water10_cluster(0)
    for n, seed in [(3, 1), (12, 2), (40, 3)]:
        yield syn.attach_synthetic_basis(syn.organic_molecule(n, seed), aux_l_max=2, seed=seed)


@pytest.mark.parametrize("k", range(4))
def test_device_pairs_match_front_end(k):
    mol = list(_molecules())[k]
    ref = pu.form_pair_data(mol, 1e-14)
    dev = dpairs.form_pair_data_device(mol, 1e-14)
    assert set(ref) == set(dev)
    for key in ref:
        r, d = ref[key], dev[key]
        assert r.coefficient.shape == d.coefficient.shape, key
        # same pairs: compare as sets keyed by (shells, exponents), then the order
        kr = np.stack([r.i_ao_start, r.j_ao_start, r.A_a[:, 3], r.B_b[:, 3]], 1)
        kd = np.stack([d.i_ao_start, d.j_ao_start, d.A_a[:, 3], d.B_b[:, 3]], 1)
        assert np.array_equal(np.unique(kr, axis=0), np.unique(kd, axis=0)), key
        np.testing.assert_allclose(d.upper_bound, r.upper_bound, rtol=1e-12, atol=0)
        same_order = np.all(kr == kd, axis=1)
        # rows can only swap among (near-)equal bounds
        assert np.all(same_order | np.isclose(r.upper_bound, d.upper_bound, rtol=1e-11, atol=0)), key
        for f in ("P_p", "A_a", "B_b", "coefficient"):
            np.testing.assert_allclose(getattr(d, f)[same_order], getattr(r, f)[same_order], rtol=1e-12,
                                       atol=1e-300)


def test_integrals_from_device_pairs():
    mol = syn.attach_synthetic_basis(syn.organic_molecule(8, 5), aux_l_max=3, seed=5)
    ad = pu.form_auxiliary_pair_data(mol)
    J_ref = mi.three_center(pu.form_pair_data(mol, 1e-14), ad, mol)
    J_dev = mi.three_center(dpairs.form_pair_data_device(mol, 1e-14), ad, mol)
    np.testing.assert_allclose(J_dev, J_ref, rtol=0, atol=1e-13)
