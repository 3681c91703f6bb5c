"""The reference's own, unchanged Python wrappers bind this library.

Where a reference checkout is present (EIP_REFERENCE_ROOT, or the location
oracle/Makefile names), a child process imports the reference's
electron_integral_playground.molecular_integral modules with LD_LIBRARY_PATH
holding only this library's directory: each module's
``ctypes.cdll.LoadLibrary("libmolecular_integral.so")`` (three_center.py:7 and
its siblings) must load this library and resolve the four entry points it
calls.  No integral is computed (there is no GPU here; the GPU test
test_gpu_reference_frontend.py makes the calls).  Also checks that the pair
tables of this repository's front end have plain-int class keys, which the
reference wrappers assert (three_center.py:19-20).
"""

import os
import pathlib
import subprocess
import sys
import textwrap

import pytest

REPO = pathlib.Path(__file__).resolve().parent.parent
LIB = REPO / "electron-integral-playground_b200" / "lib" / "libmolecular_integral.so"


def _reference_root():
    root = os.environ.get("EIP_REFERENCE_ROOT")
    if root is None:
        for line in (REPO / "oracle" / "Makefile").read_text().splitlines():
            if line.startswith("REF_ROOT ?="):
                root = line.split("?=", 1)[1].strip()
    if root and (pathlib.Path(root) / "electron_integral_playground" / "molecular_integral").is_dir():
        return root
    return None


def test_reference_wrappers_load_this_library():
    root = _reference_root()
    if root is None:
        pytest.skip("no reference checkout")
    if not LIB.exists():
        pytest.skip("library not built")
    child = textwrap.dedent('''
        import ctypes, importlib
        mods = [importlib.import_module("electron_integral_playground.molecular_integral." + n)
                for n in ("three_center", "two_center", "nuclear_attraction", "overlap")]
        maps = [l.split()[-1] for l in open("/proc/self/maps") if l.rstrip().endswith("libmolecular_integral.so")]
        print("LOADED", sorted(set(maps)))
        for m in mods:
            lib = m.libmolecular_integral
            for sym in ("three_center", "two_center", "nuclear_attraction", "overlap"):
                getattr(lib, sym)
    ''')
    env = dict(os.environ, LD_LIBRARY_PATH=str(LIB.parent), PYTHONPATH=root)
    r = subprocess.run([sys.executable, "-c", child], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("LOADED")][0]
    assert str(LIB.resolve()) in line and line.count("libmolecular_integral.so") == 1, line


def test_pair_tables_have_int_class_keys():
    import importlib

    syn = importlib.import_module("electron-integral-playground_b200.synthetic")
    pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
    mol = syn.water10_cluster(0)
    for (i, j) in pu.form_pair_data(mol, 1e-14):
        assert type(i) is int and type(j) is int
    for k in pu.form_auxiliary_pair_data(mol):
        assert type(k) is int
