"""Load the golden fixtures of tests/golden/ into front-end objects."""

import importlib
import pathlib

import numpy as np

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
ds = importlib.import_module("electron-integral-playground_b200.data_structure")


def case_names(kind=None):
    names = sorted(p.stem for p in GOLDEN.glob("test_*.npz"))
    if kind:
        names = [n for n in names if n.startswith(f"test_{kind}_")]
    return names


def _pairs(d, prefix):
    if f"{prefix}classes" not in d.files:
        return None
    out = {}
    for tag in d[f"{prefix}classes"]:
        tag = str(tag)
        key = tuple(int(x) for x in tag.split("_")) if "_" in tag else int(tag)
        g = lambda f: d[f"{prefix}{tag}__{f}"] if f"{prefix}{tag}__{f}" in d.files else None
        out[key] = ds.PrimitivePairData(P_p=g("P_p"), A_a=g("A_a"), B_b=g("B_b"), coefficient=g("coefficient"),
                                        i_ao_start=g("i_ao_start"), j_ao_start=g("j_ao_start"),
                                        i_atom=None, j_atom=None)
    return out


def _basis(d, prefix):
    out = {}
    for k in d.files:
        if k.startswith(prefix) and k.endswith("__l"):
            el = k[len(prefix):-3]
            ls, npr = d[f"{prefix}{el}__l"], d[f"{prefix}{el}__nprim"]
            e, c = d[f"{prefix}{el}__exp"], d[f"{prefix}{el}__coef"]
            shells, o = [], 0
            for l, n in zip(ls, npr):
                shells.append(ds.GaussianShell(int(l), -1, -1, e[o:o + n].copy(), c[o:o + n].copy()))
                o += n
            out[el] = shells
    return out or None


class Case:
    def __init__(self, name):
        d = np.load(GOLDEN / f"{name}.npz")
        self.name = name
        self.kind = str(d["kind"]) if "kind" in d.files else None
        self.elements = [str(x) for x in d["elements"]]
        self.geometry = d["geometry"]
        self.spherical = bool(d["spherical"]) if "spherical" in d.files else True
        self.n_ao = int(d["n_ao"]) if "n_ao" in d.files else 0
        self.n_aux = int(d["n_aux"]) if "n_aux" in d.files else 0
        self.omega = float(d["omega"]) if "omega" in d.files else 0.0
        self.pair_data = _pairs(d, "pair__")
        self.aux_data = _pairs(d, "aux__")
        self.basis = _basis(d, "basis__")
        self.aux_basis = _basis(d, "auxbasis__")
        self.charge_position = d["charge_position"] if "charge_position" in d.files else None
        self.refout_shape = tuple(d["refout_shape"]) if "refout_shape" in d.files else None
        self.refout = d["refout"] if "refout" in d.files else None
        self.refout_index = d["refout_index"] if "refout_index" in d.files else None
        self.golden = d["golden"] if "golden" in d.files else None
        self.golden_atol = float(d["golden_atol"]) if "golden_atol" in d.files else None

    def molecule(self):
        return ds.Molecule(elements=list(self.elements), geometry=self.geometry.copy(), n_ao=self.n_ao,
                           n_aux=self.n_aux, spherical_basis=self.spherical)

    def sample(self, full):
        """Values of a full output tensor at the stored sample positions."""
        full = np.asarray(full)
        return full.ravel()[self.refout_index] if self.refout_index is not None else full
