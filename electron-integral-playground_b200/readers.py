"""Minimal text readers for molecules (XYZ) and Gaussian-format basis sets.

Only what the integral path needs to be fed: the same input formats and unit
handling as the reference readers (geometry_reader/xyz_reader.py:8-41,
basis_reader/gaussian_basis_reader.py:9-93, units.py:8-9), so that tests and
synthetic generators can hand basis text to the front end exactly as the
reference's tests do.  No bundled basis-set library is shipped.
"""

from enum import Enum

import numpy as np

from .basis_utility import angular_letter_to_l_value
from .data_structure import GaussianShell, Molecule


class LengthUnits(Enum):
    BOHR = 1
    ANGSTROM = 2


bohr_to_angstrom = 5.2917721054482e-1
angstrom_to_bohr = 1.0 / bohr_to_angstrom


def read_xyz_content(lines, unit: LengthUnits = LengthUnits.ANGSTROM) -> Molecule:
    if isinstance(lines, str):
        lines = lines.split("\n")
    n_atom = int(lines[0])
    if n_atom <= 0 or len(lines) < n_atom + 2:
        raise ValueError("malformed XYZ content")
    elements, xyz = [], np.empty((n_atom, 3))
    for i in range(n_atom):
        f = lines[i + 2].split()
        if len(f) != 4:
            raise ValueError(f"malformed XYZ atom line: {lines[i + 2]!r}")
        elements.append(f[0])
        xyz[i] = [float(f[1]), float(f[2]), float(f[3])]
    if unit == LengthUnits.ANGSTROM:
        xyz *= angstrom_to_bohr
    elif unit != LengthUnits.BOHR:
        raise ValueError(f"unsupported unit {unit}")
    return Molecule(elements=elements, geometry=xyz, spherical_basis=True)


def read_basis_content(lines) -> dict:
    """Parse Gaussian-format basis text (``El 0`` / ``L nprim 1.00`` / ``****``).

    ``SP`` blocks become one s and one p shell sharing exponents.
    """
    if isinstance(lines, str):
        lines = lines.split("\n")
    basis, atom, shells = {}, None, None
    remaining, letter, rows = 0, None, None
    for line in lines:
        f = line.split()
        if not f or f[0].startswith("!"):
            continue
        if "ECP" in line:
            raise NotImplementedError("ECP not supported")
        if f[0].startswith("****"):
            if atom is None:
                raise ValueError("'****' without an element block")
            basis[atom] = shells
            atom, shells = None, None
            continue
        if shells is None:
            if len(f) != 2 or f[1] != "0":
                raise ValueError(f"expected element header, got {line!r}")
            atom, shells = f[0], []
            if atom in basis:
                raise ValueError(f"element {atom} defined twice")
            continue
        if remaining <= 0:
            if len(f) != 3 or float(f[2]) != 1.0:
                raise ValueError(f"expected shell header, got {line!r}")
            letter, remaining, rows = f[0], int(f[1]), []
            if remaining <= 0 or not (len(letter) == 1 or letter == "SP"):
                raise ValueError(f"bad shell header {line!r}")
            continue
        vals = [float(x.replace("D", "E")) for x in f]
        if vals[0] <= 0.0 or len(vals) != (3 if letter == "SP" else 2):
            raise ValueError(f"bad primitive line {line!r}")
        rows.append(vals)
        remaining -= 1
        if remaining == 0:
            r = np.array(rows)
            if letter == "SP":
                shells.append(GaussianShell(0, -1, -1, r[:, 0].copy(), r[:, 1].copy()))
                shells.append(GaussianShell(1, -1, -1, r[:, 0].copy(), r[:, 2].copy()))
            else:
                shells.append(GaussianShell(angular_letter_to_l_value(letter), -1, -1,
                                            r[:, 0].copy(), r[:, 1].copy()))
    return basis
