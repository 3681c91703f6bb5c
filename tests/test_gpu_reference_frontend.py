"""The drop-in boundary as the reference front end uses it.

The reference's Python wrappers (electron_integral_playground/molecular_integral/
{three_center,two_center,nuclear_attraction,overlap}.py:7) load the library
with ``ctypes.cdll.LoadLibrary("libmolecular_integral.so")``, found through
LD_LIBRARY_PATH, set no argtypes or restype, pass every scalar wrapped in
ctypes.c_int / c_bool / c_double and every array as ``ndarray.ctypes.data_as``
a double or int pointer, and assert a return value of 0 per class call
(three_center.py:28-48).  The wrappers themselves are not shipped here (they
are the reference's source, absent where the GPU tests run), so this test
makes the same calls in the same form from a child process whose
LD_LIBRARY_PATH holds only this library's directory, checks that the library
it loaded by that bare name is this one, and compares the four integrals of
the 10-water cluster with the reference library built from its own sources
(oracle/_ref) at 1e-12.
"""

import os
import pathlib
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

REPO = pathlib.Path(__file__).resolve().parent.parent
LIB_DIR = REPO / "electron-integral-playground_b200" / "lib"

CHILD = textwrap.dedent(r'''
    import ctypes, importlib, sys
    import numpy as np
    sys.path.insert(0, sys.argv[1])
    syn = importlib.import_module("electron-integral-playground_b200.synthetic")
    pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
    lib = ctypes.cdll.LoadLibrary("libmolecular_integral.so")
    loaded = [l.split()[-1] for l in open("/proc/self/maps") if l.rstrip().endswith("libmolecular_integral.so")]
    mol = syn.water10_cluster(0)
    pd, ad = pu.form_pair_data(mol, 1e-14), pu.form_auxiliary_pair_data(mol)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    n_ao, n_aux = mol.n_ao, mol.n_aux
    J3 = np.zeros((n_aux, n_ao, n_ao))
    for (i, j), p in pd.items():
        assert type(i) is int and type(j) is int
        for k, a in ad.items():
            assert type(k) is int
            rc = lib.three_center(ctypes.c_int(i), ctypes.c_int(j), ctypes.c_int(k), dp(p.P_p), dp(p.A_a),
                                  dp(p.B_b), dp(p.coefficient), ip(p.i_ao_start), ip(p.j_ao_start),
                                  ctypes.c_int(p.P_p.shape[0]), dp(a.A_a), dp(a.coefficient), ip(a.i_ao_start),
                                  ctypes.c_int(a.A_a.shape[0]), dp(J3), ctypes.c_int(n_ao), ctypes.c_int(n_aux),
                                  ctypes.c_bool(mol.spherical_basis), ctypes.c_double(0.0))
            assert rc == 0
    J2 = np.zeros((n_aux, n_aux))
    for i, a in ad.items():
        for j, b in ad.items():
            if i > j:
                continue
            rc = lib.two_center(ctypes.c_int(i), ctypes.c_int(j), dp(a.A_a), dp(a.coefficient), ip(a.i_ao_start),
                                ctypes.c_int(a.A_a.shape[0]), dp(b.A_a), dp(b.coefficient), ip(b.i_ao_start),
                                ctypes.c_int(b.A_a.shape[0]), dp(J2), ctypes.c_int(n_aux),
                                ctypes.c_bool(mol.spherical_basis), ctypes.c_double(0.0))
            assert rc == 0
    C = np.ascontiguousarray(mol.geometry, dtype=np.float64)
    V = np.zeros((n_ao, n_ao, C.shape[0]))
    S = np.zeros((n_ao, n_ao))
    for (i, j), p in pd.items():
        rc = lib.nuclear_attraction(ctypes.c_int(i), ctypes.c_int(j), dp(p.P_p), dp(p.A_a), dp(p.B_b),
                                    dp(p.coefficient), ip(p.i_ao_start), ip(p.j_ao_start),
                                    ctypes.c_int(p.P_p.shape[0]), dp(C), ctypes.c_int(C.shape[0]), dp(V),
                                    ctypes.c_int(n_ao), ctypes.c_bool(mol.spherical_basis), ctypes.c_double(0.0))
        assert rc == 0
        rc = lib.overlap(ctypes.c_int(i), ctypes.c_int(j), dp(p.A_a), dp(p.B_b), dp(p.coefficient),
                         ip(p.i_ao_start), ip(p.j_ao_start), ctypes.c_int(p.P_p.shape[0]), dp(S),
                         ctypes.c_int(n_ao), ctypes.c_bool(mol.spherical_basis))
        assert rc == 0
    np.savez(sys.argv[2], J3=J3, J2=J2, V=V, S=S, loaded=np.array(loaded))
''')


def test_reference_calling_convention_through_ld_library_path(tmp_path):
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference library not built (make -C oracle ref)")
    script = tmp_path / "frontend_calls.py"
    script.write_text(CHILD)
    out = tmp_path / "out.npz"
    env = dict(os.environ, LD_LIBRARY_PATH=str(LIB_DIR))
    subprocess.run([sys.executable, str(script), str(REPO), str(out)], env=env, check=True, timeout=900)
    got = np.load(out)
    loaded = {pathlib.Path(p).resolve() for p in got["loaded"]}
    assert loaded == {(LIB_DIR / "libmolecular_integral.so").resolve()}

    import importlib

    syn = importlib.import_module("electron-integral-playground_b200.synthetic")
    pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
    mol = syn.water10_cluster(0)
    pd, ad = pu.form_pair_data(mol, 1e-14), pu.form_auxiliary_pair_data(mol)
    want = {"J3": oracle.drive_three_center(ref, pd, ad, mol), "J2": oracle.drive_two_center(ref, ad, mol),
            "V": oracle.drive_nuclear_attraction(ref, pd, mol, np.asarray(mol.geometry)),
            "S": oracle.drive_overlap(ref, pd, mol)}
    for k, w in want.items():
        # (P|Q) reaches ~1e2: 1e-12 absolute up to |v| = 10, 1e-13 relative above
        tol = np.maximum(1e-12, 1e-13 * np.abs(w)) if k == "J2" else 1e-12
        err = np.abs(got[k] - w)
        assert np.all(err <= tol), (k, float(err.max()))
