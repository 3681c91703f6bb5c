"""Lattice-summed integrals on the GPU against the reference library on the
same image lists: the short-range (erfc) three-centre integrals and nuclear
attraction, and the Gamma-point overlap, for a water molecule in a triclinic
cell."""

import importlib
import math

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

syn = importlib.import_module("electron-integral-playground_b200.synthetic")
per = importlib.import_module("electron-integral-playground_b200.periodic")
pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
ds = importlib.import_module("electron-integral-playground_b200.data_structure")

OMEGA, PAIR_R, AUX_R = 0.5, 20.0, 15.0


@pytest.fixture(scope="module")
def crystal():
    mol = syn.water_cluster(1, 2.0, seed=4)
    syn.attach_synthetic_basis(mol, aux_l_max=2, seed=4)
    b = 1.8897261246
    cell = per.get_cell_from_lattice_constant(5.0 * b, 5.5 * b, 6.0 * b, math.radians(90), math.radians(95),
                                              math.radians(100))
    return ds.Crystal(cell=cell, atoms=mol)


def _ref():
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference library not built")
    return ref


def test_lattice_three_center_short_range(crystal):
    ref = _ref()
    mol = crystal.atoms
    ad = pu.form_auxiliary_pair_data(mol)
    got = per.lattice_three_center_sr(crystal, ad, OMEGA, PAIR_R, AUX_R)
    images = per.image_pair_data(crystal, per.lattice_offsets(crystal.cell, PAIR_R))
    aux = per.image_auxiliary_pair_data(crystal, ad, per.lattice_offsets(crystal.cell, AUX_R))
    parts = [sum(oracle.drive_three_center(ref, pd, aux, mol, omega=w) for _, pd in images) for w in (0.0, OMEGA)]
    want = parts[0] - parts[1]
    scale = max(1.0, float(np.abs(parts[0]).max()))
    err = float(np.abs(got - want).max())
    assert err <= 1e-12 * scale, (err, scale)


def test_lattice_nuclear_attraction_short_range(crystal):
    ref = _ref()
    mol = crystal.atoms
    got = per.lattice_nuclear_attraction_sr(crystal, OMEGA, PAIR_R, AUX_R)
    images = per.image_pair_data(crystal, per.lattice_offsets(crystal.cell, PAIR_R))
    q = per.image_charges(crystal, per.lattice_offsets(crystal.cell, AUX_R))
    parts = [sum(oracle.drive_nuclear_attraction(ref, pd, mol, q, omega=w) for _, pd in images)
             for w in (0.0, OMEGA)]
    n_atom = len(mol.geometry)
    want = (parts[0] - parts[1]).reshape(mol.n_ao, mol.n_ao, -1, n_atom).sum(axis=2)
    scale = max(1.0, float(np.abs(parts[0]).max()))
    assert float(np.abs(got - want).max()) <= 1e-12 * scale


def test_gamma_point_overlap(crystal):
    ref = _ref()
    mol = crystal.atoms
    got = per.lattice_overlap(crystal, PAIR_R)
    images = per.image_pair_data(crystal, per.lattice_offsets(crystal.cell, PAIR_R))
    want = sum(oracle.drive_overlap(ref, pd, mol) for _, pd in images)
    assert float(np.abs(got - want).max()) <= 1e-12
    assert float(np.abs(got - got.T).max()) <= 1e-13
