"""S through the CUDA library; mirrors the reference overlap.py:7-32."""

import numpy as np

from .._lib import as_f64, as_i32, check, dp, ip, lib


def overlap(pair_data, molecule) -> np.ndarray:
    n_ao = molecule.n_ao
    if n_ao <= 0:
        raise ValueError("molecule needs an orbital basis")
    S = np.zeros((n_ao, n_ao), dtype=np.float64, order="C")
    L = lib()
    for (li, lj), p in pair_data.items():
        A, B = as_f64(p.A_a, (4,)), as_f64(p.B_b, (4,))
        c, ia, ja = as_f64(p.coefficient), as_i32(p.i_ao_start), as_i32(p.j_ao_start)
        if A.shape[0] == 0:
            continue
        rc = L.overlap(int(li), int(lj), dp(A), dp(B), dp(c), ip(ia), ip(ja), A.shape[0], dp(S), n_ao,
                       bool(molecule.spherical_basis))
        check(rc, f"overlap({li},{lj})")
    return S
