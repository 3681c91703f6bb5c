"""CPU references for the integral path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package, and only to check or time against it; the product path
never calls it.

* ``oracle`` -- ``oracle/lib/liboracle.so``, the plain-C restatement of the
  reference drivers (md_oracle.c; parity pinned against the reference's
  golden vectors and against the reference library itself).
* ``reference`` -- ``oracle/_ref/libmolecular_integral.so``, the reference's
  own C++/OpenMP sources compiled unmodified by ``make -C oracle ref``.

``drive_*`` run the per-class loop of the reference front end
(electron_integral_playground/molecular_integral/*.py) over either library.
"""

import ctypes
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ORACLE_SO = HERE / "lib" / "liboracle.so"
REFERENCE_SO = HERE / "_ref" / "libmolecular_integral.so"

_c_double_p = ctypes.POINTER(ctypes.c_double)
_c_int_p = ctypes.POINTER(ctypes.c_int)


def _dp(a):
    return a.ctypes.data_as(_c_double_p)


def _ip(a):
    return a.ctypes.data_as(_c_int_p)


class IntegralLibrary:
    """The four C entry points of one library (names optionally prefixed)."""

    def __init__(self, path, prefix=""):
        self.path = str(path)
        self.lib = ctypes.CDLL(self.path)
        self.three_center_fn = getattr(self.lib, prefix + "three_center")
        self.two_center_fn = getattr(self.lib, prefix + "two_center")
        self.nuclear_attraction_fn = getattr(self.lib, prefix + "nuclear_attraction")
        self.overlap_fn = getattr(self.lib, prefix + "overlap")
        for f in (self.three_center_fn, self.two_center_fn, self.nuclear_attraction_fn, self.overlap_fn):
            f.restype = ctypes.c_int


_cache = {}


def oracle():
    if "oracle" not in _cache:
        if not ORACLE_SO.exists():
            raise FileNotFoundError(f"{ORACLE_SO} missing: run `make -C oracle`")
        _cache["oracle"] = IntegralLibrary(ORACLE_SO, "oracle_")
        lib = _cache["oracle"].lib
        lib.oracle_boys.argtypes = [ctypes.c_int, ctypes.c_double, _c_double_p]
        lib.oracle_boys_many.argtypes = [ctypes.c_int, ctypes.c_int, _c_double_p, _c_double_p]
        lib.oracle_spherical_matrix.argtypes = [ctypes.c_int, _c_double_p]
    return _cache["oracle"]


def reference():
    """The reference library, or None when it was not built here."""
    if "reference" not in _cache:
        _cache["reference"] = IntegralLibrary(REFERENCE_SO) if REFERENCE_SO.exists() else None
    return _cache["reference"]


def boys(L, x):
    y = np.empty(L + 1)
    oracle().lib.oracle_boys(int(L), float(x), _dp(y))
    return y


def boys_many(L, xs):
    """F_m(x), m = 0..L, for every x (long-double series): shape (len(xs), L + 1)."""
    xs = np.ascontiguousarray(xs, dtype=np.float64)
    y = np.empty((xs.size, L + 1))
    oracle().lib.oracle_boys_many(int(L), int(xs.size), _dp(xs), _dp(y))
    return y


def spherical_matrix(l):
    out = np.empty((2 * l + 1, (l + 1) * (l + 2) // 2))
    oracle().lib.oracle_spherical_matrix(int(l), _dp(out))
    return out


def call_three_center(lib, li, lj, lk, pair, aux, out, n_ao, n_aux, spherical, omega):
    return lib.three_center_fn(ctypes.c_int(li), ctypes.c_int(lj), ctypes.c_int(lk),
                               _dp(pair.P_p), _dp(pair.A_a), _dp(pair.B_b), _dp(pair.coefficient),
                               _ip(pair.i_ao_start), _ip(pair.j_ao_start), ctypes.c_int(pair.P_p.shape[0]),
                               _dp(aux.A_a), _dp(aux.coefficient), _ip(aux.i_ao_start),
                               ctypes.c_int(aux.A_a.shape[0]), _dp(out), ctypes.c_int(n_ao),
                               ctypes.c_int(n_aux), ctypes.c_bool(spherical), ctypes.c_double(omega))


def drive_three_center(lib, pair_data, aux_data, molecule, omega=0.0, out=None):
    out = np.zeros((molecule.n_aux, molecule.n_ao, molecule.n_ao)) if out is None else out
    for (li, lj), pair in pair_data.items():
        for lk, aux in aux_data.items():
            rc = call_three_center(lib, li, lj, lk, pair, aux, out, molecule.n_ao, molecule.n_aux,
                                   molecule.spherical_basis, omega)
            assert rc == 0
    return out


def drive_two_center(lib, aux_data, molecule, omega=0.0):
    out = np.zeros((molecule.n_aux, molecule.n_aux))
    for li, a in aux_data.items():
        for lj, b in aux_data.items():
            if li > lj:
                continue
            rc = lib.two_center_fn(ctypes.c_int(li), ctypes.c_int(lj), _dp(a.A_a), _dp(a.coefficient),
                                   _ip(a.i_ao_start), ctypes.c_int(a.A_a.shape[0]), _dp(b.A_a),
                                   _dp(b.coefficient), _ip(b.i_ao_start), ctypes.c_int(b.A_a.shape[0]),
                                   _dp(out), ctypes.c_int(molecule.n_aux),
                                   ctypes.c_bool(molecule.spherical_basis), ctypes.c_double(omega))
            assert rc == 0
    return out


def drive_nuclear_attraction(lib, pair_data, molecule, charge_position, omega=0.0):
    cp = np.ascontiguousarray(charge_position, dtype=np.float64)
    out = np.zeros((molecule.n_ao, molecule.n_ao, cp.shape[0]))
    for (li, lj), p in pair_data.items():
        rc = lib.nuclear_attraction_fn(ctypes.c_int(li), ctypes.c_int(lj), _dp(p.P_p), _dp(p.A_a),
                                       _dp(p.B_b), _dp(p.coefficient), _ip(p.i_ao_start),
                                       _ip(p.j_ao_start), ctypes.c_int(p.P_p.shape[0]), _dp(cp),
                                       ctypes.c_int(cp.shape[0]), _dp(out), ctypes.c_int(molecule.n_ao),
                                       ctypes.c_bool(molecule.spherical_basis), ctypes.c_double(omega))
        assert rc == 0
    return out


def drive_overlap(lib, pair_data, molecule):
    out = np.zeros((molecule.n_ao, molecule.n_ao))
    for (li, lj), p in pair_data.items():
        rc = lib.overlap_fn(ctypes.c_int(li), ctypes.c_int(lj), _dp(p.A_a), _dp(p.B_b), _dp(p.coefficient),
                            _ip(p.i_ao_start), _ip(p.j_ao_start), ctypes.c_int(p.P_p.shape[0]), _dp(out),
                            ctypes.c_int(molecule.n_ao), ctypes.c_bool(molecule.spherical_basis))
        assert rc == 0
    return out


def set_reference_threads(n):
    """OpenMP threads of the reference library's parallel loops in this
    process (the library is already loaded, so the environment variable alone
    would not reach it: set the runtime's default thread count as well)."""
    os.environ["OMP_NUM_THREADS"] = str(n)
    try:
        ctypes.CDLL("libgomp.so.1").omp_set_num_threads(ctypes.c_int(int(n)))
        return True
    except OSError:
        return False


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or None."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None
