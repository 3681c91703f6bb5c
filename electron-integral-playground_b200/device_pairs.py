"""Screened orbital pair tables built on the device (``eip_pairs_*``).

Same tables as :func:`pair_utility.form_pair_data` (the reference front end's
construction, pair_utility.py:6-188) — the same pairs, bounds and order, with
row values that can differ from numpy's in the last bit (device exp/pow) —
computed by CUDA kernels: one thread per shell pair for the bounds, a
device compaction and stable radix sort by descending bound, one thread per
row for the table values.
"""

import ctypes

import numpy as np

from ._lib import IntegralError, as_f64, as_i32, dp, ip, lib
from .data_structure import Molecule, PrimitivePairData

_vp = ctypes.c_void_p


def _bind(L):
    if getattr(L, "_pairs_bound", False):
        return
    _dpp, _ipp = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    L.eip_pairs_build.argtypes = [ctypes.c_int, _ipp, _ipp, _ipp, _ipp, _dpp, _dpp, ctypes.c_int, _dpp,
                                  ctypes.c_double]
    L.eip_pairs_build.restype = _vp
    L.eip_pairs_error.argtypes = [_vp]
    L.eip_pairs_error.restype = ctypes.c_char_p
    L.eip_pairs_count.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
    L.eip_pairs_copy.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _dpp, _dpp, _dpp, _dpp, _ipp, _ipp, _ipp, _ipp,
                                 _dpp]
    L.eip_pairs_destroy.argtypes = [_vp]
    L.eip_pairs_destroy.restype = None
    L._pairs_bound = True


def form_pair_data_device(molecule: Molecule, schwarz_upper_bound: float = 1e-14) -> dict:
    """{(l_i, l_j): PrimitivePairData} like pair_utility.form_pair_data."""
    shells = molecule.basis_shells
    if not shells or molecule.n_ao <= 0:
        raise ValueError("molecule has no orbital basis attached")
    L = lib()
    _bind(L)
    sl = as_i32([s.angular for s in shells])
    sa = as_i32([s.i_atom for s in shells])
    so = as_i32([s.i_ao_start for s in shells])
    sn = as_i32([len(s.primitive_exponents) for s in shells])
    pe = as_f64(np.concatenate([np.asarray(s.primitive_exponents, np.float64) for s in shells]))
    pc = as_f64(np.concatenate([np.asarray(s.primitive_coefficients, np.float64) for s in shells]))
    geom = as_f64(np.asarray(molecule.geometry, np.float64).reshape(-1, 3), (3,))
    h = L.eip_pairs_build(len(shells), ip(sl), ip(sa), ip(so), ip(sn), dp(pe), dp(pc), geom.shape[0], dp(geom),
                          float(schwarz_upper_bound))
    if not h:
        raise IntegralError("eip_pairs_build failed")
    try:
        err = L.eip_pairs_error(h).decode(errors="replace")
        if err:
            raise IntegralError(f"eip_pairs_build: {err}")
        out = {}
        ls = sorted({int(s.angular) for s in shells})
        for li in ls:
            for lj in ls:
                if li > lj:
                    continue
                n = L.eip_pairs_count(h, li, lj)
                if n <= 0:
                    continue
                P, A, B = np.empty((n, 4)), np.empty((n, 4)), np.empty((n, 4))
                c, bnd = np.empty(n), np.empty(n)
                ia, ja, iat, jat = (np.empty(n, np.int32) for _ in range(4))
                rc = L.eip_pairs_copy(h, li, lj, dp(P), dp(A), dp(B), dp(c), ip(ia), ip(ja), ip(iat), ip(jat),
                                      dp(bnd))
                if rc != 0:
                    raise IntegralError(f"eip_pairs_copy: status {rc}")
                out[(li, lj)] = PrimitivePairData(P_p=P, A_a=A, B_b=B, coefficient=c, i_ao_start=ia, j_ao_start=ja,
                                                  i_atom=iat, j_atom=jat, upper_bound=bnd)
        return out
    finally:
        L.eip_pairs_destroy(h)
