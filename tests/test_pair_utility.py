"""The host pair builder against the reference front end: pair counts of the
reference's own test (tests/test_pair_utility.py:24,46) and bit-identical
pair tables for every golden case."""

import importlib

import numpy as np
import pytest

from golden_cases import GOLDEN, Case, case_names, _basis, _pairs

pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
bu = importlib.import_module("electron-integral-playground_b200.basis_utility")
ds = importlib.import_module("electron-integral-playground_b200.data_structure")

REF_COUNTS = {
    "pair_counts_compact": {(0, 0): 171, (0, 1): 158, (0, 2): 36, (1, 1): 51, (1, 2): 18, (2, 2): 3},
    "pair_counts_sparse": {(0, 0): 144, (0, 1): 142, (0, 2): 34, (1, 1): 47, (1, 2): 18, (2, 2): 3},
}


def build(elements, geometry, basis, spherical=True):
    mol = ds.Molecule(elements=list(elements), geometry=np.array(geometry), spherical_basis=spherical)
    bu.attach_basis_to_molecule(mol, basis)
    return mol


@pytest.mark.parametrize("name", sorted(REF_COUNTS))
def test_pair_counts(name):
    d = np.load(GOLDEN / f"{name}.npz")
    mol = build([str(x) for x in d["elements"]], d["geometry"], _basis(d, "basis__"))
    lst = pu.form_primitive_pair_list(mol, 1e-14)
    assert {k: len(v[0]) for k, v in lst.items()} == REF_COUNTS[name]
    for k, v in lst.items():
        bnd = v[4]
        assert np.all(bnd[:-1] >= bnd[1:]) and np.all(bnd >= 1e-14)
    mine = pu.form_pair_data(mol, 1e-14)
    ref = _pairs(d, "pair__")
    for k in ref:
        for f in ("P_p", "A_a", "B_b", "coefficient", "i_ao_start", "j_ao_start"):
            assert np.array_equal(getattr(mine[k], f), getattr(ref[k], f)), (k, f)


@pytest.mark.parametrize("name", [n for n in case_names() if "two_center" not in n])
def test_pair_tables_bit_identical(name):
    c = Case(name)
    mol = build(c.elements, c.geometry, c.basis, c.spherical)
    assert mol.n_ao == c.n_ao
    mine = pu.form_pair_data(mol, 1e-14)
    assert list(mine) == list(c.pair_data) or set(mine) == set(c.pair_data)
    for k, ref in c.pair_data.items():
        for f in ("P_p", "A_a", "B_b", "coefficient", "i_ao_start", "j_ao_start"):
            assert np.array_equal(getattr(mine[k], f), getattr(ref, f)), (k, f)
    if c.aux_basis is not None:
        bu.attach_auxiliary_basis_to_molecule(mol, c.aux_basis)
        assert mol.n_aux == c.n_aux
        aux = pu.form_auxiliary_pair_data(mol)
        for k, ref in c.aux_data.items():
            for f in ("A_a", "coefficient", "i_ao_start"):
                assert np.array_equal(getattr(aux[k], f), getattr(ref, f)), (k, f)


def test_synthetic_generators_terminate_and_respect_geometry():
    syn = importlib.import_module("electron-integral-playground_b200.synthetic")
    for seed in range(40):
        for n in (1, 3, 7, 25):
            m = syn.organic_molecule(n, seed)
            assert len(m.elements) == n
            if n > 1:
                d = np.linalg.norm(m.geometry[:, None] - m.geometry[None], axis=-1) * 0.52917721054482
                assert np.min(d[np.triu_indices(n, 1)]) > 0.9
    w = syn.water_cluster(10, 9.0, 0)
    o = w.geometry[0::3] * 0.52917721054482
    d = np.linalg.norm(o[:, None] - o[None], axis=-1)
    assert np.min(d[np.triu_indices(10, 1)]) >= 2.6


def test_normalize_shell_matches_reference_on_bundled_bases():
    """normalize_shell against the reference's on every H/C/N/O/F shell of the
    reference's bundled orbital and auxiliary basis sets (fixture made by
    tests/golden/make_golden.py): bit for bit."""
    import pathlib
    from copy import deepcopy

    bu = importlib.import_module("electron-integral-playground_b200.basis_utility")
    ds = importlib.import_module("electron-integral-playground_b200.data_structure")
    f = np.load(pathlib.Path(__file__).parent / "golden" / "normalize_shell.npz")
    n = int(f["n"])
    assert n > 100
    for k in range(n):
        s = ds.GaussianShell(angular=int(f[f"l_{k}"]), i_ao_start=-1, i_atom=-1,
                             primitive_exponents=f[f"exp_{k}"].copy(), primitive_coefficients=f[f"raw_{k}"].copy())
        t = deepcopy(s)
        bu.normalize_shell(t)
        np.testing.assert_array_equal(t.primitive_exponents, f[f"exp_{k}"])
        np.testing.assert_array_equal(t.primitive_coefficients, f[f"norm_{k}"], err_msg=f"shell {k}")
