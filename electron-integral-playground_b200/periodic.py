"""Periodic (lattice-summed) integrals over the same kernels.

The reference declares the periodic types (Cell, Crystal, PeriodicPrimitivePair,
electron_integral_playground/data_structure.py:49-66) and builds a cell from
lattice constants (cell_utility.py:7-28), but computes no periodic integral.
This module computes the lattice sums that are finite term by term, each as a
sum of molecular-ABI integrals over explicit image lists, so that the
reference library evaluated on the same lists is their oracle:

* the Gamma-point overlap  S_{mu nu} = sum_T < mu_0 | nu_T >;
* the short-range (erfc) three-centre integrals
      (mu nu|P)^{sr} = sum_{T, T'} (mu_0 nu_T | erfc(omega r)/r | P_{T'}),
  computed as the Coulomb minus the erf-attenuated integrals (both in the
  reference ABI: omega = 0 and omega > 0, MI/three_center.cpp:46-49), which is
  the lattice-convergent part of a range-separated density fitting;
* the short-range nuclear attraction  V_{mu nu}(C) = sum_{T, T'}
  (mu_0 nu_T | erfc(omega r)/r | C_{T'}) per atom C of the cell.

Image lists: orbital pairs (shell i in the home cell, shell j in cell T) are
screened with the front end's pair bound (pair_utility.py rule) for every T
of the cell's images within a radius, in the reference's i <= j shell order
with its mirroring of (mu, nu) into (nu, mu).  The converged sums are
invariant under a common translation of all images (the mirror of
(mu_0 nu_T | P_T') is (nu_0 mu_{-T} | P_{T'-T})), so there the mirroring is
exact; with truncated image sets the result is what the reference computes on
the same lists, and its (mu, nu) asymmetry measures how far the auxiliary
radius is from convergence (it must reach past the pair images' centres by
the operator's range).  Auxiliary images are extra
primitives of the same auxiliary function (same first index), so the kernels
contract them into one output like primitives of a contracted shell; charge
images are extra charges whose columns are summed.

Every image T of the orbital pairs is one molecule slot of a batch (a shell
pair's primitive pairs must share one AB vector), so one batch launch computes
all images.
"""

import math

import numpy as np

from .data_structure import Cell, Crystal, PrimitivePairData
from .pair_utility import REFERENCE_PAIR_THRESHOLD, form_primitive_pair_data, form_primitive_pair_list


def get_cell_from_lattice_constant(a: float, b: float, c: float, alpha: float, beta: float, gamma: float,
                                   dimension: int = 3) -> Cell:
    """Cell from lattice constants (a, b, c in Bohr; alpha, beta, gamma in
    radians): the first vector along x, the second in the xy plane, the third
    completing the triclinic cell (reference cell_utility.py:7-28); 3D only."""
    if dimension not in (1, 2, 3):
        raise ValueError("dimension must be 1, 2 or 3")
    if dimension != 3:
        raise NotImplementedError("only 3D periodic cells are supported")
    ca, cb, cg, sg = math.cos(alpha), math.cos(beta), math.cos(gamma), math.sin(gamma)
    volume = a * b * c * math.sqrt(1.0 - ca * ca - cb * cb - cg * cg + 2.0 * ca * cb * cg)
    R = np.zeros((3, 3))
    R[0, 0] = a
    R[1, 0], R[1, 1] = b * cg, b * sg
    R[2, 0] = c * cb
    R[2, 1] = c * (ca - cb * cg) / sg
    R[2, 2] = volume / (a * b * sg)
    return Cell(dimension=dimension, lattice_vectors=R)


def lattice_offsets(cell: Cell, radius: float) -> np.ndarray:
    """Integer image offsets n (rows) whose displacement n @ lattice_vectors is
    within `radius` Bohr, the home cell first, then by increasing length."""
    R = np.asarray(cell.lattice_vectors, dtype=np.float64)
    # a box of integer offsets that contains the sphere
    inv = np.linalg.inv(R)
    n_max = np.ceil(radius * np.linalg.norm(inv, axis=0)).astype(int) + 1
    grid = np.stack(np.meshgrid(*[np.arange(-k, k + 1) for k in n_max], indexing="ij"), -1).reshape(-1, 3)
    disp = grid @ R
    d = np.linalg.norm(disp, axis=1)
    keep = d <= radius + 1e-12
    grid, d = grid[keep], d[keep]
    order = np.lexsort((grid[:, 2], grid[:, 1], grid[:, 0], d))
    return grid[order]


def image_pair_data(crystal: Crystal, offsets, threshold: float = REFERENCE_PAIR_THRESHOLD) -> list:
    """[(offset, pair tables)] for every image offset with at least one
    screened pair: shell i in the home cell, shell j displaced by the offset."""
    R = np.asarray(crystal.cell.lattice_vectors, dtype=np.float64)
    out = []
    for n in np.asarray(offsets, dtype=int):
        shift = n @ R
        plist = form_primitive_pair_list(crystal.atoms, threshold, j_shift=None if not n.any() else shift)
        if plist:
            out.append((tuple(int(x) for x in n),
                        form_primitive_pair_data(crystal.atoms, plist, j_shift=None if not n.any() else shift)))
    return out


def image_auxiliary_pair_data(crystal: Crystal, aux_data: dict, offsets) -> dict:
    """The auxiliary tables with every primitive repeated at each image offset
    (same first function: the images add into one output function)."""
    R = np.asarray(crystal.cell.lattice_vectors, dtype=np.float64)
    shifts = np.asarray(offsets, dtype=int) @ R
    out = {}
    for l, a in aux_data.items():
        A = np.asarray(a.A_a, dtype=np.float64)
        rows = np.concatenate([np.c_[A[:, :3] + s[None, :], A[:, 3]] for s in shifts])
        out[l] = PrimitivePairData(
            P_p=None, A_a=np.ascontiguousarray(rows), B_b=None,
            coefficient=np.ascontiguousarray(np.tile(np.asarray(a.coefficient), len(shifts))),
            i_ao_start=np.ascontiguousarray(np.tile(np.asarray(a.i_ao_start, dtype=np.int32), len(shifts))),
            j_ao_start=None,
            i_atom=None if a.i_atom is None else np.tile(np.asarray(a.i_atom, dtype=np.int32), len(shifts)),
            j_atom=None)
    return out


def image_charges(crystal: Crystal, offsets) -> np.ndarray:
    """Positions of every atom at every image offset, (n_offset * n_atom, 3),
    offset-major (column c of the result belongs to atom c % n_atom)."""
    R = np.asarray(crystal.cell.lattice_vectors, dtype=np.float64)
    geom = np.asarray(crystal.atoms.geometry, dtype=np.float64)
    shifts = np.asarray(offsets, dtype=int) @ R
    return np.ascontiguousarray(np.concatenate([geom + s[None, :] for s in shifts]))


def _crystal_batch(bt, crystal, images, aux, omega, precision, charges=None):
    mols = [crystal.atoms] * len(images)
    pds = [pd for _, pd in images]
    b = bt.ThreeCenterBatch(mols, pds, [aux] * len(images), omega=omega, precision=precision,
                            charges_list=None if charges is None else [charges] * len(images))
    b.alloc_output()
    b.run()
    b.status()
    return b


def lattice_three_center_sr(crystal: Crystal, aux_data: dict, omega: float, pair_radius: float,
                            aux_radius: float, precision: str = "fp64"):
    """(mu nu|P)^{sr} = sum_{T, T'} (mu_0 nu_T | erfc(omega r)/r | P_{T'}) as a dense
    (n_aux, n_ao, n_ao) array (the reference's three-centre layout and
    mirroring): orbital pair images within pair_radius (screened), auxiliary
    images within aux_radius; the Coulomb batch minus the erf-attenuated batch
    over the same image lists, one molecule slot per orbital image."""
    from . import batch as bt

    if not omega > 0.0:
        raise ValueError("the short-range operator needs omega > 0")
    images = image_pair_data(crystal, lattice_offsets(crystal.cell, pair_radius))
    aux = image_auxiliary_pair_data(crystal, aux_data, lattice_offsets(crystal.cell, aux_radius))
    mol = crystal.atoms
    out = np.zeros((mol.n_aux, mol.n_ao, mol.n_ao))
    for w, sign in ((0.0, 1.0), (omega, -1.0)):
        b = _crystal_batch(bt, crystal, images, aux, w, precision)
        for m in range(len(images)):
            out += sign * b.dense(m)
        b.close()
    return out


def lattice_nuclear_attraction_sr(crystal: Crystal, omega: float, pair_radius: float, charge_radius: float):
    """V_{mu nu}(C) = sum_{T, T'} (mu_0 nu_T | erfc(omega r)/r | C_{T'}) for every atom
    C of the cell, (n_ao, n_ao, n_atom), unit charges (not scaled by -Z)."""
    from . import batch as bt

    if not omega > 0.0:
        raise ValueError("the short-range operator needs omega > 0")
    images = image_pair_data(crystal, lattice_offsets(crystal.cell, pair_radius))
    charges = image_charges(crystal, lattice_offsets(crystal.cell, charge_radius))
    mol = crystal.atoms
    n_atom = len(mol.geometry)
    V = np.zeros((mol.n_ao, mol.n_ao, charges.shape[0]))
    aux = {}  # no auxiliary basis: the point charges are the only ket class
    for w, sign in ((0.0, 1.0), (omega, -1.0)):
        b = bt.ThreeCenterBatch([mol] * len(images), [pd for _, pd in images], [aux] * len(images), omega=w,
                                charges_list=[charges] * len(images))
        b.alloc_output()
        b.run()
        b.status()
        for m in range(len(images)):
            V += sign * b.dense_V(m)
        b.close()
    return V.reshape(mol.n_ao, mol.n_ao, -1, n_atom).sum(axis=2)


def lattice_overlap(crystal: Crystal, pair_radius: float):
    """Gamma-point overlap S_{mu nu} = sum_T < mu_0 | nu_T > (n_ao, n_ao), through
    the drop-in overlap entry point per image."""
    from .molecular_integral import overlap

    mol = crystal.atoms
    S = np.zeros((mol.n_ao, mol.n_ao))
    for _, pd in image_pair_data(crystal, lattice_offsets(crystal.cell, pair_radius)):
        S += overlap(pd, mol)
    return S
