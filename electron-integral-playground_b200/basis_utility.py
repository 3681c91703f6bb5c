"""Basis-set attachment and contraction normalisation.

Behaviour follows the reference front end
(electron_integral_playground/basis_utility.py:24-140): shells are normalised
on their pure-x Cartesian component, atoms are laid out atom-leading, and the
auxiliary basis shares the orbital basis' ``spherical_basis`` flag.  The
arithmetic of :func:`normalize_shell` is kept in the same order as the
reference so that the coefficients, and hence every pair table built from
them, are bit-identical to the reference's.
"""

from copy import deepcopy
from math import factorial

import numpy as np

from .data_structure import GaussianShell, Molecule

ANGULAR_LETTERS = "SPDFGHIKLM"


def angular_letter_to_l_value(letter: str) -> int:
    letter = letter.upper()
    if len(letter) != 1 or letter not in ANGULAR_LETTERS:
        raise ValueError(f"unknown angular momentum letter {letter!r}")
    return ANGULAR_LETTERS.index(letter)


def n_ao_of_angular(l: int, spherical: bool = True) -> int:
    return 2 * l + 1 if spherical else (l + 1) * (l + 2) // 2


def normalize_shell(shell: GaussianShell) -> None:
    """Scale ``shell.primitive_coefficients`` so that <x^L|x^L> = 1.

    Primitive normalisation a^(L/2+3/4) first, then the contracted norm
        N^-2 = pi^1.5 (2L)!/(4^L L!) sum_mn c_m c_n (a_m+a_n)^(-L-3/2)
    (reference: basis_utility.py:85-140).  Not idempotent: call once per shell.
    """
    L = int(shell.angular)
    if L < 0:
        raise ValueError("negative angular momentum")
    e = np.asarray(shell.primitive_exponents, dtype=np.float64)
    c = np.asarray(shell.primitive_coefficients, dtype=np.float64)
    if e.ndim != 1 or e.shape != c.shape or e.shape[0] == 0:
        raise ValueError("shell needs matching 1-D exponent and coefficient arrays")
    c = c * np.power(e, L * 0.5 + 0.75)
    pref = np.power(np.pi, 1.5) * factorial(2 * L) / (4 ** L * factorial(L))
    s = np.power(e[:, None] + e[None, :], -L - 1.5)
    norm = np.power(pref * np.sum(np.outer(c, c) * s), -0.5)
    c *= norm
    shell.primitive_coefficients = c


def assign_ao_index_to_shell(molecule: Molecule) -> None:
    """Atom-leading AO offsets for the orbital and auxiliary shell lists."""

    def _assign(shells, spherical):
        shells.sort(key=lambda s: s.i_atom)  # stable: keeps file order per atom
        offset = 0
        for s in shells:
            s.i_ao_start = offset
            offset += n_ao_of_angular(s.angular, spherical)
        return offset

    done = False
    if molecule.basis_shells:
        molecule.n_ao = _assign(molecule.basis_shells, molecule.spherical_basis)
        done = True
    if molecule.auxiliary_basis_shells:
        molecule.n_aux = _assign(molecule.auxiliary_basis_shells, molecule.spherical_basis)
        done = True
    if not done:
        raise ValueError("molecule has no shells to index")


def attach_basis_to_molecule(molecule: Molecule, basis_set: dict, if_auxiliary_basis: bool = False) -> None:
    used = {}
    for element in molecule.elements:
        if element not in basis_set:
            raise KeyError(f"basis set has no entry for element {element}")
        if element not in used:
            used[element] = deepcopy(basis_set[element])
    for shells in used.values():
        for s in shells:
            normalize_shell(s)

    target = []
    for i_atom, element in enumerate(molecule.elements):
        for s in deepcopy(used[element]):
            s.i_atom = i_atom
            target.append(s)
    if if_auxiliary_basis:
        molecule.auxiliary_basis_shells = target
    else:
        molecule.basis_shells = target
    assign_ao_index_to_shell(molecule)


def attach_auxiliary_basis_to_molecule(molecule: Molecule, basis_set: dict) -> None:
    attach_basis_to_molecule(molecule, basis_set, True)
