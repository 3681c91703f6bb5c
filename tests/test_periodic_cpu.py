"""Periodic front end on the CPU: the cell from lattice constants, the image
offsets, and the image pair tables (no device needed)."""

import importlib
import math

import numpy as np

syn = importlib.import_module("electron-integral-playground_b200.synthetic")
per = importlib.import_module("electron-integral-playground_b200.periodic")
pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
ds = importlib.import_module("electron-integral-playground_b200.data_structure")


def _crystal():
    mol = syn.water_cluster(1, 2.0, seed=4)
    syn.attach_synthetic_basis(mol, aux_l_max=2, seed=4)
    b = 1.8897261246
    cell = per.get_cell_from_lattice_constant(5.0 * b, 5.5 * b, 6.0 * b, math.radians(90), math.radians(95),
                                              math.radians(100))
    return ds.Crystal(cell=cell, atoms=mol)


def test_cell_vectors_have_the_lattice_constants():
    a, b, c = 7.0, 8.0, 9.0
    al, be, ga = math.radians(80), math.radians(85), math.radians(95)
    R = per.get_cell_from_lattice_constant(a, b, c, al, be, ga).lattice_vectors
    np.testing.assert_allclose(np.linalg.norm(R, axis=1), [a, b, c], rtol=1e-14)
    cos = lambda u, v: u @ v / np.linalg.norm(u) / np.linalg.norm(v)
    np.testing.assert_allclose([cos(R[1], R[2]), cos(R[0], R[2]), cos(R[0], R[1])],
                               [math.cos(al), math.cos(be), math.cos(ga)], atol=1e-14)
    assert R[0, 1] == R[0, 2] == R[1, 2] == 0.0
    cube = per.get_cell_from_lattice_constant(3.0, 3.0, 3.0, math.pi / 2, math.pi / 2, math.pi / 2).lattice_vectors
    np.testing.assert_allclose(cube, 3.0 * np.eye(3), atol=1e-15)


def test_lattice_offsets_cover_the_sphere_symmetrically():
    cell = _crystal().cell
    off = per.lattice_offsets(cell, 20.0)
    assert tuple(off[0]) == (0, 0, 0)
    d = np.linalg.norm(off @ cell.lattice_vectors, axis=1)
    assert np.all(d <= 20.0 + 1e-12) and np.all(np.diff(d) >= -1e-12)
    keys = {tuple(x) for x in off}
    assert all(tuple(-x) in keys for x in off)  # every image comes with its inverse
    # nothing within the radius is missing
    g = np.stack(np.meshgrid(*[np.arange(-6, 7)] * 3, indexing="ij"), -1).reshape(-1, 3)
    inside = {tuple(x) for x in g[np.linalg.norm(g @ cell.lattice_vectors, axis=1) <= 20.0]}
    assert inside == keys


def test_home_image_pairs_equal_the_molecular_pairs():
    cr = _crystal()
    images = per.image_pair_data(cr, per.lattice_offsets(cr.cell, 20.0))
    assert images[0][0] == (0, 0, 0)
    mol_pd = pu.form_pair_data(cr.atoms, 1e-14)
    for key, p in images[0][1].items():
        for f in ("P_p", "A_a", "B_b", "coefficient", "i_ao_start", "j_ao_start"):
            np.testing.assert_array_equal(getattr(p, f), getattr(mol_pd[key], f))
    # an image's B centres are the home atoms displaced by the image vector
    R = cr.cell.lattice_vectors
    for n, pd in images[1:]:
        shift = np.asarray(n) @ R
        for p in pd.values():
            np.testing.assert_allclose(p.B_b[:, :3] - shift, np.asarray(cr.atoms.geometry)[p.j_atom], atol=1e-12)
    # both an image and its inverse are present whenever one is
    keys = {n for n, _ in images}
    assert all(tuple(-np.asarray(n)) in keys for n in keys)
