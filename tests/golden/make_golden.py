"""Regenerate the golden fixtures in tests/golden/ from the reference.

Run in a container that has the reference checkout and its library built by
``make -C oracle ref``::

    python tests/golden/make_golden.py [--reference <reference checkout>]

(default: $EIP_REFERENCE_ROOT).

For every integral test of the reference (electron_integral_playground/
molecular_integral/tests/test_*_integral.py) the script runs the test
function unmodified, with the front-end integral call and the final
``assert_allclose`` intercepted, and records:

* the molecule (elements, Bohr geometry, spherical flag) and the raw,
  un-normalised orbital / auxiliary basis per element as the test defined it;
* omega and point charges;
* the reference front end's pair tables (the exact C-ABI inputs);
* ``golden``: the PySCF values the test compares against, when the reference
  still ships that file (several large ones are missing upstream);
* ``refout``: the reference library's own output on these inputs (subsampled
  with ``refout_index`` when the tensor is large).

It also records the two pair-list count tests of tests/test_pair_utility.py.
Fixtures are small .npz files; nothing here runs at test time.
"""

import argparse
import ctypes
import importlib
import os
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
REPO = HERE.parent.parent
MAX_FULL = 20000  # store full outputs up to this many elements, else subsample


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("EIP_REFERENCE_ROOT"))
    args = ap.parse_args()
    if not args.reference or not (pathlib.Path(args.reference) / "electron_integral_playground").is_dir():
        sys.exit("make_golden: give the reference checkout with --reference or EIP_REFERENCE_ROOT")
    ref_lib_dir = REPO / "oracle" / "_ref"
    if str(ref_lib_dir) not in os.environ.get("LD_LIBRARY_PATH", ""):
        # The reference wrappers dlopen("libmolecular_integral.so") at import.
        env = dict(os.environ, LD_LIBRARY_PATH=f"{ref_lib_dir}:{os.environ.get('LD_LIBRARY_PATH', '')}")
        os.execve(sys.executable, [sys.executable] + sys.argv, env)
    sys.path.insert(0, args.reference)
    ctypes.CDLL(str(ref_lib_dir / "libmolecular_integral.so"))

    import electron_integral_playground.basis_utility as rbu

    recorded = {}

    def raw_basis(basis_set):
        out = {}
        for el, shells in basis_set.items():
            out[el] = [(int(s.angular), np.array(s.primitive_exponents, dtype=np.float64),
                        np.array(s.primitive_coefficients, dtype=np.float64)) for s in shells]
        return out

    orig_attach = rbu.attach_basis_to_molecule

    def capture_attach(molecule, basis_set, if_auxiliary_basis=False):
        key = "aux_basis" if if_auxiliary_basis else "basis"
        recorded[key] = raw_basis(basis_set)
        recorded["elements"] = list(molecule.elements)
        recorded["geometry"] = np.array(molecule.geometry, dtype=np.float64)
        return orig_attach(molecule, basis_set, if_auxiliary_basis)

    def capture_aux_attach(molecule, basis_set):
        return capture_attach(molecule, basis_set, True)

    cases = []
    for kind in ("three_center", "two_center", "nuclear_attraction", "overlap"):
        mod = importlib.import_module(f"electron_integral_playground.molecular_integral.tests.test_{kind}_integral")
        wrapper = getattr(mod, kind)

        def make_capture(kind=kind, wrapper=wrapper):
            def capture(*a, **kw):
                out = wrapper(*a, **kw)
                names = {"three_center": ["pair_data", "aux_data", "molecule", "omega"],
                         "two_center": ["aux_data", "molecule", "omega"],
                         "nuclear_attraction": ["pair_data", "molecule", "charge_position", "omega"],
                         "overlap": ["pair_data", "molecule"]}[kind]
                bound = dict(zip(names, a))
                bound.update(kw)
                recorded["call"] = bound
                recorded["refout"] = out
                return out
            return capture

        class NpProxy:
            def __init__(self):
                self.testing = self

            def __getattr__(self, name):
                return getattr(np, name)

            def assert_allclose(self, actual, desired, rtol=0, atol=0):
                recorded["golden"] = np.array(desired)
                recorded["atol"] = atol

        setattr(mod, kind, make_capture())
        mod.attach_basis_to_molecule = capture_attach
        if hasattr(mod, "attach_auxiliary_basis_to_molecule"):
            mod.attach_auxiliary_basis_to_molecule = capture_aux_attach
        mod.np = NpProxy()
        for name in sorted(n for n in dir(mod) if n.startswith("test_")):
            recorded.clear()
            try:
                getattr(mod, name)()
                status = "golden"
            except FileNotFoundError:
                status = "no-golden"
            cases.append((kind, name, status, dict(recorded)))
            print(f"{kind:20s} {name:50s} {status}", flush=True)

    for kind, name, status, rec in cases:
        save_case(kind, name, status, rec)
    save_pair_counts(args.reference)
    save_normalisation(args.reference)


def pack_pairs(prefix, table, out):
    keys = []
    for key, d in table.items():
        tag = f"{key[0]}_{key[1]}" if isinstance(key, tuple) else f"{key}"
        keys.append(tag)
        for f in ("P_p", "A_a", "B_b", "coefficient", "i_ao_start", "j_ao_start"):
            v = getattr(d, f)
            if v is not None:
                out[f"{prefix}{tag}__{f}"] = np.asarray(v)
    out[f"{prefix}classes"] = np.array(keys)


def pack_basis(prefix, basis, out):
    # Per element: shell angular momenta, primitive counts, concatenated
    # exponents and coefficients (file order).
    for el, shells in basis.items():
        out[f"{prefix}{el}__l"] = np.array([l for l, _, _ in shells], dtype=np.int32)
        out[f"{prefix}{el}__nprim"] = np.array([len(e) for _, e, _ in shells], dtype=np.int32)
        out[f"{prefix}{el}__exp"] = np.concatenate([e for _, e, _ in shells])
        out[f"{prefix}{el}__coef"] = np.concatenate([c for _, _, c in shells])


def save_case(kind, name, status, rec):
    call = rec["call"]
    mol = call["molecule"]
    out = {
        "kind": np.array(kind), "name": np.array(name),
        "elements": np.array(rec["elements"]), "geometry": rec["geometry"],
        "spherical": np.array(bool(mol.spherical_basis)),
        "n_ao": np.array(mol.n_ao), "n_aux": np.array(mol.n_aux),
        "omega": np.array(float(call.get("omega", 0.0))),
    }
    if "basis" in rec:
        pack_basis("basis__", rec["basis"], out)
    if "aux_basis" in rec:
        pack_basis("auxbasis__", rec["aux_basis"], out)
    if "pair_data" in call:
        pack_pairs("pair__", call["pair_data"], out)
    if "aux_data" in call:
        pack_pairs("aux__", call["aux_data"], out)
    if "charge_position" in call:
        out["charge_position"] = np.asarray(call["charge_position"], dtype=np.float64)
    refout = np.asarray(rec["refout"])
    out["refout_shape"] = np.array(refout.shape)
    if refout.size <= MAX_FULL:
        out["refout"] = refout
    else:
        rng = np.random.default_rng(0)
        idx = np.sort(rng.choice(refout.size, size=MAX_FULL, replace=False))
        out["refout_index"] = idx
        out["refout"] = refout.ravel()[idx]
    if status == "golden":
        golden = np.asarray(rec["golden"]).reshape(refout.shape)
        out["golden_atol"] = np.array(rec["atol"])
        if golden.size <= MAX_FULL:
            out["golden"] = golden
        else:
            out["golden"] = golden.ravel()[out["refout_index"]]
    np.savez_compressed(HERE / f"{name}.npz", **out)


def save_pair_counts(reference):
    from electron_integral_playground.basis_reader.gaussian_basis_reader import read_basis
    from electron_integral_playground.geometry_reader.xyz_reader import read_xyz_content
    from electron_integral_playground.basis_utility import attach_basis_to_molecule
    from electron_integral_playground.pair_utility import form_pair_data

    geometries = {
        "pair_counts_compact": "3\n\nO 0 0 0\nH 1 0 0\nF -0.8 0.2 0\n",
        "pair_counts_sparse": "3\n\nO 0 0 0\nH 3 0 0\nF -0.8 2.2 0\n",
    }
    basis = read_basis("def2-svp")
    for name, xyz in geometries.items():
        mol = read_xyz_content(xyz)
        out = {"elements": np.array(mol.elements), "geometry": np.array(mol.geometry)}
        pack_basis("basis__", {el: [(int(s.angular), np.array(s.primitive_exponents),
                                     np.array(s.primitive_coefficients)) for s in basis[el]]
                               for el in set(mol.elements)}, out)
        attach_basis_to_molecule(mol, basis)
        pack_pairs("pair__", form_pair_data(mol, 1e-14), out)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print("pair counts", name)


def save_normalisation(reference):
    """normalize_shell on every shell of the bundled orbital and auxiliary
    basis sets for H, C, N, O, F (the reference's own basis library)."""
    from copy import deepcopy

    from electron_integral_playground.basis_reader.gaussian_basis_reader import read_basis
    from electron_integral_playground.basis_utility import normalize_shell

    out = {}
    k = 0
    data = pathlib.Path(reference) / "electron_integral_playground" / "data" / "basis_sets"
    names = sorted(p.name.split(".")[0] for p in data.iterdir() if p.name.endswith(".basis"))
    for basis_name in names:
        try:
            basis = read_basis(basis_name)
        except Exception as exc:  # a basis the reference does not bundle
            print("skip", basis_name, exc)
            continue
        for el in ("H", "C", "N", "O", "F"):
            for s in basis.get(el, []):
                t = deepcopy(s)
                normalize_shell(t)
                out[f"l_{k}"] = np.array(int(s.angular))
                out[f"exp_{k}"] = np.array(s.primitive_exponents, dtype=np.float64)
                out[f"raw_{k}"] = np.array(s.primitive_coefficients, dtype=np.float64)
                out[f"norm_{k}"] = np.array(t.primitive_coefficients, dtype=np.float64)
                k += 1
    out["n"] = np.array(k)
    np.savez_compressed(HERE / "normalize_shell.npz", **out)
    print("normalize_shell shells", k)


if __name__ == "__main__":
    main()
