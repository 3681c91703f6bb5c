"""Data types of the integral front end.

Mirrors the reference's dataclasses field by field
(electron_integral_playground/data_structure.py:6-47) so that code written
against the reference front end reads the same here.  Arrays follow the same
conventions: positions in Bohr, (n, 4) rows of ``[x, y, z, exponent]``,
C-contiguous float64, AO offsets as int32.
"""

from dataclasses import dataclass, field
from typing import Optional

import numpy as np


@dataclass
class GaussianShell:
    angular: int
    i_ao_start: int
    i_atom: int
    primitive_exponents: np.ndarray
    primitive_coefficients: np.ndarray


BasisSet = dict  # element symbol -> list[GaussianShell]


@dataclass
class Molecule:
    elements: list
    geometry: np.ndarray  # Bohr, (n_atom, 3)
    basis_shells: Optional[list] = None
    n_ao: int = 0
    auxiliary_basis_shells: Optional[list] = None
    n_aux: int = 0
    spherical_basis: bool = True


@dataclass
class PrimitivePairData:
    """Structure-of-arrays table of primitive shell pairs of one (l_i, l_j) class.

    Same fields as the reference's PrimitivePairData
    (electron_integral_playground/data_structure.py:36-45).  For an auxiliary
    table only ``A_a``, ``coefficient``, ``i_ao_start`` and ``i_atom`` are set.
    """
    P_p: Optional[np.ndarray]
    A_a: np.ndarray
    B_b: Optional[np.ndarray]
    coefficient: np.ndarray
    i_ao_start: np.ndarray
    j_ao_start: Optional[np.ndarray]
    i_atom: np.ndarray
    j_atom: Optional[np.ndarray]
    # Not in the reference: the screening bound of each primitive pair, kept so
    # that device-side triplet screening can use it (the C ABI never sees it).
    upper_bound: Optional[np.ndarray] = field(default=None, repr=False)


PrimitivePairDataAngularList = dict  # (l_i, l_j) or l -> PrimitivePairData


@dataclass
class Cell:
    """A periodic cell (reference data_structure.py:49-52): each row of
    lattice_vectors is one lattice vector, in Bohr."""
    dimension: int
    lattice_vectors: np.ndarray


@dataclass
class Crystal:
    """Reference data_structure.py:54-57: the cell and the atoms of one image
    (absolute positions of an arbitrary image of each atom), with their basis
    sets attached as for a molecule."""
    cell: Cell
    atoms: Molecule


@dataclass
class PeriodicPrimitivePair:
    """Reference data_structure.py:59-66: a primitive pair whose j primitive
    sits in the image cell displaced by cell_offset (3 integers) lattice vectors."""
    i_shell: int
    j_shell: int
    i_primitive: int
    j_primitive: int
    cell_offset: np.ndarray
    upper_bound: float
