"""Seeded synthetic molecules and basis sets for the benchmark workloads.

No public benchmark suite exists for this path; these generators stand in for
real chemistry with the shapes, sizes and value ranges the workloads name:

* ``water_cluster(n_water, box_angstrom, seed)`` -- rigid waters (O-H 0.96 A,
  H-O-H 104.5 deg), uniform random centres in a cube, uniform random
  orientation (unit quaternion), O-O distance >= 2.6 A by rejection.
* ``organic_molecule(n_atom, seed)`` -- H/C/N/O (0.5/0.3/0.1/0.1) grown by
  random bonded placement within valences (C 4, N 3, O 2): X-H 1.09 A,
  heavy-heavy U[1.40, 1.54] A, non-bonded distances >= 2.0 A (geminal 1-3
  pairs >= 1.6 A).
* ``orbital_basis_text(elements, seed)`` -- Gaussian-format text; O/C/N get
  3s2p1d and H 2s1p.  Every shell draws 1-6 distinct exponents (uniform count)
  from an even-tempered ladder of ratio 3.0 starting at 0.12 and capped at
  5000 (heavy s) / 30 (H s), the cap shrinking by 10x per unit of angular
  momentum; contraction coefficients are U[0.1, 1] before normalisation.
* ``auxiliary_basis_text(elements, l_max)`` -- uncontracted even-tempered
  shells, ratio 2.5 from 0.1 up to 200 (9 exponents per l), l = 0..l_max.

All sizes in Angstrom on input; molecules are returned in Bohr like the XYZ
reader does.
"""

import math

import numpy as np

from .basis_utility import ANGULAR_LETTERS, attach_auxiliary_basis_to_molecule, attach_basis_to_molecule
from .data_structure import Molecule
from .readers import angstrom_to_bohr, read_basis_content

OH_ANGSTROM = 0.96
HOH_DEGREES = 104.5


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def water_cluster(n_water: int, box_angstrom: float, seed: int = 0, min_oo: float = 2.6) -> Molecule:
    rng = np.random.default_rng(seed)
    half = math.radians(HOH_DEGREES) / 2
    local = np.array([[0.0, 0.0, 0.0],
                      [OH_ANGSTROM * math.sin(half), 0.0, OH_ANGSTROM * math.cos(half)],
                      [-OH_ANGSTROM * math.sin(half), 0.0, OH_ANGSTROM * math.cos(half)]])
    centres = []
    tries = 0
    while len(centres) < n_water:
        tries += 1
        if tries > 1000000:
            raise RuntimeError("could not place waters; box too small")
        c = rng.uniform(0.0, box_angstrom, size=3)
        if all(np.linalg.norm(c - o) >= min_oo for o in centres):
            centres.append(c)
    xyz, elements = [], []
    for c in centres:
        R = _random_rotation(rng)
        for el, r in zip(("O", "H", "H"), local):
            xyz.append(c + R @ r)
            elements.append(el)
    return Molecule(elements=elements, geometry=np.array(xyz) * angstrom_to_bohr, spherical_basis=True)


_VALENCE = {"C": 4, "N": 3, "O": 2}


def _place(rng, xyz, neighbours, parent, bond):
    """Random direction around `parent` keeping non-bonded distances >= 2.0 A
    (>= 1.6 A to the parent's other neighbours); relaxes both floors by 10 %
    after every 200 failed directions, so it always terminates."""
    floor_nb, floor_gem = 2.0, 1.6
    for _ in range(50):
        for _ in range(200):
            v = rng.normal(size=3)
            pos = xyz[parent] + bond * v / np.linalg.norm(v)
            gem = set(neighbours[parent])
            if all(k == parent or np.linalg.norm(pos - xyz[k]) >= (floor_gem if k in gem else floor_nb)
                   for k in range(len(xyz))):
                return pos
        floor_nb *= 0.9
        floor_gem *= 0.9
    return pos


def organic_molecule(n_atom: int, seed: int = 0) -> Molecule:
    """Grow a molecule by random bonded placement (see module docstring).

    Composition is drawn first (H/C/N/O 0.5/0.3/0.1/0.1, first atom heavy);
    hydrogens beyond the skeleton's free valences (C 4, N 3, O 2) become carbon.
    The heavy-atom tree is grown first, then hydrogens fill free valences.
    """
    if n_atom < 1:
        raise ValueError("n_atom must be >= 1")
    rng = np.random.default_rng(seed)
    symbols = np.array(["H", "C", "N", "O"])
    probs = np.array([0.5, 0.3, 0.1, 0.1])
    heavy_probs = probs[1:] / probs[1:].sum()
    elems = [str(rng.choice(symbols[1:], p=heavy_probs))] + [str(rng.choice(symbols, p=probs))
                                                               for _ in range(n_atom - 1)]
    while True:
        heavy = [e for e in elems if e != "H"]
        capacity = sum(_VALENCE[e] for e in heavy) - 2 * (len(heavy) - 1)
        n_h = len(elems) - len(heavy)
        if n_h <= capacity:
            break
        elems[elems.index("H")] = "C"
    heavy = [e for e in elems if e != "H"]
    elements, xyz, neighbours, free = [heavy[0]], [np.zeros(3)], [[]], [_VALENCE[heavy[0]]]
    for el in heavy[1:]:
        # keep a free valence on the tree for every heavy atom still to come
        cand = [i for i in range(len(elements)) if free[i] >= 2] or [i for i in range(len(elements)) if free[i] >= 1]
        parent = cand[rng.integers(len(cand))]
        pos = _place(rng, xyz, neighbours, parent, rng.uniform(1.40, 1.54))
        elements.append(el)
        xyz.append(pos)
        neighbours.append([parent])
        neighbours[parent].append(len(xyz) - 1)
        free.append(_VALENCE[el] - 1)
        free[parent] -= 1
    for _ in range(len(elems) - len(heavy)):
        cand = [i for i in range(len(elements)) if elements[i] != "H" and free[i] >= 1]
        parent = cand[rng.integers(len(cand))]
        pos = _place(rng, xyz, neighbours, parent, 1.09)
        elements.append("H")
        xyz.append(pos)
        neighbours.append([parent])
        neighbours[parent].append(len(xyz) - 1)
        free.append(0)
        free[parent] -= 1
    return Molecule(elements=elements, geometry=np.array(xyz) * angstrom_to_bohr, spherical_basis=True)


_SHELLS = {"H": (2, 1, 0), "C": (3, 2, 1), "N": (3, 2, 1), "O": (3, 2, 1)}
_S_CAP = {"H": 30.0, "C": 5000.0, "N": 5000.0, "O": 5000.0}


def _ladder(start, ratio, cap):
    out = []
    e = start
    while e <= cap * (1 + 1e-12):
        out.append(e)
        e *= ratio
    return out


def orbital_basis_text(elements, seed: int = 0) -> str:
    rng = np.random.default_rng(seed + 7919)
    lines = []
    for el in sorted(set(elements)):
        lines.append(f"{el}     0")
        counts = _SHELLS[el]
        for l, n_shell in enumerate(counts):
            ladder = _ladder(0.12, 3.0, max(_S_CAP[el] / 10.0 ** l, 0.5))
            for _ in range(n_shell):
                k = int(rng.integers(1, 7))
                k = min(k, len(ladder))
                chosen = sorted(rng.choice(ladder, size=k, replace=False), reverse=True)
                lines.append(f"{ANGULAR_LETTERS[l]}    {k}   1.00")
                for e in chosen:
                    lines.append(f"    {float(e)!r}    {float(rng.uniform(0.1, 1.0))!r}")
        lines.append("****")
    return "\n".join(lines) + "\n"


def auxiliary_basis_text(elements, l_max: int) -> str:
    ladder = _ladder(0.1, 2.5, 200.0)
    lines = []
    for el in sorted(set(elements)):
        lines.append(f"{el}     0")
        for l in range(l_max + 1):
            for e in ladder:
                lines.append(f"{ANGULAR_LETTERS[l]}    1   1.00")
                lines.append(f"    {float(e)!r}    1.0")
        lines.append("****")
    return "\n".join(lines) + "\n"


def attach_synthetic_basis(molecule: Molecule, aux_l_max: int, seed: int = 0, spherical: bool = True) -> Molecule:
    molecule.spherical_basis = spherical
    attach_basis_to_molecule(molecule, read_basis_content(orbital_basis_text(["H", "C", "N", "O"], seed)))
    attach_auxiliary_basis_to_molecule(molecule, read_basis_content(auxiliary_basis_text(["H", "C", "N", "O"], aux_l_max)))
    return molecule


def water10_cluster(seed: int = 0) -> Molecule:
    """10 waters in a 9 A cube; aux s-f."""
    return attach_synthetic_basis(water_cluster(10, 9.0, seed), aux_l_max=3, seed=seed)


def water100_cluster(seed: int = 0) -> Molecule:
    """100 waters in a 15 A cube; aux s-f."""
    return attach_synthetic_basis(water_cluster(100, 15.0, seed), aux_l_max=3, seed=seed)


def molecule_sizes(n_molecule: int, lo: int, hi: int, seed: int):
    rng = np.random.default_rng(seed + 104729)
    return [int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))))) for _ in range(n_molecule)]


def organic_batch(seed: int = 0, n_molecule: int = 64):
    """64 organic molecules of 3-60 atoms (log-uniform); aux s-g."""
    sizes = molecule_sizes(n_molecule, 3, 60, seed)
    return [attach_synthetic_basis(organic_molecule(n, seed * 1000 + i), aux_l_max=4, seed=seed)
            for i, n in enumerate(sizes)]


def random_shell_triplet(rng, l_orbital_max=4, l_aux_max=5, max_primitives=8, box_angstrom=6.0,
                         exponent_range=(0.05, 1e4)):
    """One random shell triplet (l_i <= l_j | l_k): centres uniform in a cube,
    1..max_primitives primitives per shell, exponents log-uniform, coefficients
    uniform in [0.1, 1].  Returns ((l_i, l_j), pair table, l_k, aux table,
    molecule stub with n_ao = n_i + n_j and n_aux = n_k, spherical)."""
    from .data_structure import PrimitivePairData

    li, lj = (int(x) for x in sorted(rng.integers(0, l_orbital_max + 1, size=2)))
    lk = int(rng.integers(0, l_aux_max + 1))
    A, B, C = rng.uniform(0, box_angstrom, size=(3, 3)) * angstrom_to_bohr
    npi, npj, npk = (int(x) for x in rng.integers(1, max_primitives + 1, size=3))
    lo, hi = np.log(exponent_range[0]), np.log(exponent_range[1])
    ea, eb, ek = (np.exp(rng.uniform(lo, hi, n)) for n in (npi, npj, npk))
    ca, cb, ck = rng.uniform(0.1, 1, npi), rng.uniform(0.1, 1, npj), rng.uniform(0.1, 1, npk)
    a, b = np.repeat(ea, npj), np.tile(eb, npi)
    p = a + b
    P = (a[:, None] * A + b[:, None] * B) / p[:, None]
    coef = np.repeat(ca, npj) * np.tile(cb, npi) * np.exp(-a * b / p * np.sum((A - B) ** 2))
    n_i, n_k = 2 * li + 1, 2 * lk + 1
    pair = PrimitivePairData(P_p=np.ascontiguousarray(np.c_[P, p]),
                             A_a=np.ascontiguousarray(np.c_[np.tile(A, (len(a), 1)), a]),
                             B_b=np.ascontiguousarray(np.c_[np.tile(B, (len(a), 1)), b]), coefficient=coef,
                             i_ao_start=np.zeros(len(a), np.int32), j_ao_start=np.full(len(a), n_i, np.int32),
                             i_atom=None, j_atom=None)
    aux = PrimitivePairData(P_p=None, A_a=np.ascontiguousarray(np.c_[np.tile(C, (npk, 1)), ek]), B_b=None,
                            coefficient=ck, i_ao_start=np.zeros(npk, np.int32), j_ao_start=None, i_atom=None,
                            j_atom=None)
    mol = Molecule(elements=[], geometry=np.zeros((0, 3)), n_ao=n_i + 2 * lj + 1, n_aux=n_k, spherical_basis=True)
    return (li, lj), pair, lk, aux, mol


def random_shell_triplets(seed: int = 0, n: int = 2000):
    """2000 random shell triplets: centres in a 6 A cube, orbital l <= 4,
    auxiliary l <= 5, 1-8 primitives, exponents log-uniform in [0.05, 1e4]."""
    rng = np.random.default_rng(seed + 3)
    return [random_shell_triplet(rng) for _ in range(n)]
