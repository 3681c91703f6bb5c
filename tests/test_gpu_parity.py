"""GPU parity of the drop-in C ABI against the reference.

Every call goes through libmolecular_integral.so's reference-compatible entry
points (via the package's ctypes front end).  References:
* the reference library itself, compiled from its sources into oracle/_ref/
  (run on the same inputs, on the host cores), at 1e-12 absolute -- the bar
  for the plain FP64 path;
* the PySCF golden vectors shipped with the reference tests, at those tests'
  own tolerances (test_*_integral.py:17-18);
* the C oracle for random high-angular-momentum triplets.
"""

import importlib

import numpy as np
import pytest

import oracle
from golden_cases import Case, case_names

pytestmark = pytest.mark.gpu

mi = importlib.import_module("electron-integral-playground_b200.molecular_integral")
lib = importlib.import_module("electron-integral-playground_b200._lib")
syn = importlib.import_module("electron-integral-playground_b200.synthetic")
pu = importlib.import_module("electron-integral-playground_b200.pair_utility")

FP64_ATOL = 1e-12


def run_gpu(c):
    mol = c.molecule()
    if c.kind == "three_center":
        return mi.three_center(c.pair_data, c.aux_data, mol, c.omega)
    if c.kind == "two_center":
        return mi.two_center(c.aux_data, mol, c.omega)
    if c.kind == "nuclear_attraction":
        return mi.nuclear_attraction(c.pair_data, mol, c.charge_position, c.omega)
    return mi.overlap(c.pair_data, mol)


@pytest.mark.parametrize("name", case_names())
def test_golden_case(name):
    c = Case(name)
    out = run_gpu(c)
    assert out.shape == c.refout_shape
    np.testing.assert_allclose(c.sample(out), c.refout, rtol=0, atol=FP64_ATOL)
    if c.golden is not None:
        np.testing.assert_allclose(c.sample(out), c.golden, rtol=0, atol=c.golden_atol)


@pytest.fixture(scope="module")
def water10():
    mol = syn.water10_cluster(0)
    return mol, pu.form_pair_data(mol, 1e-14), pu.form_auxiliary_pair_data(mol)


def _reference_or_skip():
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference library not built (make -C oracle ref)")
    return ref


def test_water10_overlap_and_nuclear(water10):
    mol, pd, ad = water10
    ref = _reference_or_skip()
    S = mi.overlap(pd, mol)
    np.testing.assert_allclose(S, oracle.drive_overlap(ref, pd, mol), rtol=0, atol=FP64_ATOL)
    charges = mol.geometry
    V = mi.nuclear_attraction(pd, mol, charges)
    np.testing.assert_allclose(V, oracle.drive_nuclear_attraction(ref, pd, mol, charges), rtol=0, atol=FP64_ATOL)


def test_water10_two_center(water10):
    mol, pd, ad = water10
    ref = _reference_or_skip()
    J2 = mi.two_center(ad, mol)
    R2 = oracle.drive_two_center(ref, ad, mol)
    # (P|Q) reaches ~1e2 here; the reference's own Boys table is accurate to
    # ~5e-14 relative (c_library/boys_function.hpp:71), so compare at 1e-12
    # absolute where |value| <= 10 and 1e-13 relative above.
    scale = np.maximum(1.0, np.abs(R2) / 10.0)
    assert np.max(np.abs(J2 - R2) / scale) < FP64_ATOL
    np.testing.assert_allclose(J2, J2.T, rtol=0, atol=1e-14)


def test_water10_three_center(water10):
    mol, pd, ad = water10
    ref = _reference_or_skip()
    J3 = mi.three_center(pd, ad, mol)
    R3 = oracle.drive_three_center(ref, pd, ad, mol)
    np.testing.assert_allclose(J3, R3, rtol=0, atol=FP64_ATOL)
    # diagonal shell blocks are symmetric to rounding only (as in the reference)
    np.testing.assert_allclose(J3, J3.transpose(0, 2, 1), rtol=0, atol=1e-14)


def test_water10_three_center_omega(water10):
    mol, pd, ad = water10
    ref = _reference_or_skip()
    sub = {k: v for k, v in ad.items() if k <= 1}
    J3 = mi.three_center(pd, sub, mol, 0.3)
    R3 = oracle.drive_three_center(ref, pd, sub, mol, 0.3)
    np.testing.assert_allclose(J3, R3, rtol=0, atol=FP64_ATOL)


def test_device_boys_against_series():
    rng = np.random.default_rng(1)
    T = np.concatenate([[0.0, 1e-300, 1e-12, 0.025, 35.99, 36.0, 36.01, 200.0],
                        rng.uniform(0, 1, 2000), rng.uniform(0, 40, 4000), rng.uniform(0, 200, 2000)])
    L = 21
    F = lib.device_boys(L, T)
    ref = np.array([oracle.boys(L, t) for t in T])
    rel = np.abs(F - ref) / np.abs(ref)
    assert np.max(rel) < 5e-15, np.max(rel)


def test_random_high_angular_triplets():
    """Random high-angular-momentum shell triplets (orbital l <= 4, aux l <= 5,
    1-8 primitives, exponents log-uniform in [0.05, 1e4]) against the oracle."""
    ds = importlib.import_module("electron-integral-playground_b200.data_structure")
    rng = np.random.default_rng(3)
    for trial in range(24):
        li, lj = sorted(rng.integers(0, 5, size=2))
        lk = int(rng.integers(0, 6))
        centres = rng.uniform(0, 6.0, size=(3, 3)) / 0.52917721054482
        npi, npj, npk = rng.integers(1, 9, size=3)
        ea = np.exp(rng.uniform(np.log(0.05), np.log(1e4), npi))
        eb = np.exp(rng.uniform(np.log(0.05), np.log(1e4), npj))
        ek = np.exp(rng.uniform(np.log(0.05), np.log(1e4), npk))
        ca, cb, ck = rng.uniform(0.1, 1, npi), rng.uniform(0.1, 1, npj), rng.uniform(0.1, 1, npk)
        A, B, C = centres
        a, b = np.repeat(ea, npj), np.tile(eb, npi)
        p = a + b
        P = (a[:, None] * A + b[:, None] * B) / p[:, None]
        coef = np.repeat(ca, npj) * np.tile(cb, npi) * np.exp(-a * b / p * np.sum((A - B) ** 2))
        n_i, n_j, n_k = 2 * li + 1, 2 * lj + 1, 2 * lk + 1
        pair = ds.PrimitivePairData(
            P_p=np.ascontiguousarray(np.c_[P, p]), A_a=np.ascontiguousarray(np.tile(np.r_[A, 0], (len(a), 1))),
            B_b=np.ascontiguousarray(np.tile(np.r_[B, 0], (len(a), 1))), coefficient=coef,
            i_ao_start=np.zeros(len(a), np.int32), j_ao_start=np.full(len(a), n_i, np.int32),
            i_atom=None, j_atom=None)
        pair.A_a[:, 3], pair.B_b[:, 3] = a, b
        aux = ds.PrimitivePairData(P_p=None, A_a=np.ascontiguousarray(np.c_[np.tile(C, (npk, 1)), ek]), B_b=None,
                                   coefficient=ck, i_ao_start=np.zeros(npk, np.int32), j_ao_start=None,
                                   i_atom=None, j_atom=None)
        mol = ds.Molecule(elements=[], geometry=np.zeros((0, 3)), n_ao=n_i + n_j, n_aux=n_k, spherical_basis=True)
        got = mi.three_center({(int(li), int(lj)): pair}, {lk: aux}, mol)
        want = oracle.drive_three_center(oracle.oracle(), {(int(li), int(lj)): pair}, {lk: aux}, mol)
        scale = max(1.0, float(np.max(np.abs(want))))
        assert np.max(np.abs(got - want)) <= 1e-12 * scale, (trial, li, lj, lk, np.max(np.abs(got - want)), scale)
