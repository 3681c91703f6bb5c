"""(P|Q) through the CUDA library; mirrors the reference two_center.py:9-43."""

import numpy as np

from .._lib import as_f64, as_i32, check, dp, ip, lib


def two_center(pair_data, molecule, omega: float = 0.0) -> np.ndarray:
    if omega < 0.0:
        raise ValueError("omega must be >= 0")
    n_aux = molecule.n_aux
    if n_aux <= 0:
        raise ValueError("molecule needs an auxiliary basis")
    J2c = np.zeros((n_aux, n_aux), dtype=np.float64, order="C")
    L = lib()
    for li, a in pair_data.items():
        for lj, b in pair_data.items():
            if li > lj:
                continue
            A, ca, ia = as_f64(a.A_a, (4,)), as_f64(a.coefficient), as_i32(a.i_ao_start)
            B, cb, ib = as_f64(b.A_a, (4,)), as_f64(b.coefficient), as_i32(b.i_ao_start)
            if A.shape[0] == 0 or B.shape[0] == 0:
                continue
            rc = L.two_center(int(li), int(lj), dp(A), dp(ca), ip(ia), A.shape[0], dp(B), dp(cb), ip(ib), B.shape[0],
                              dp(J2c), n_aux, bool(molecule.spherical_basis), float(omega))
            check(rc, f"two_center({li}|{lj})")
    return J2c
