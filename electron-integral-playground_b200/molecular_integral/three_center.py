"""(mu nu|P) through the CUDA library; mirrors the reference three_center.py:9-51."""

import numpy as np

from .._lib import as_f64, as_i32, check, dp, ip, lib


def three_center(pair_data, auxiliary_pair_data, molecule, omega: float = 0.0) -> np.ndarray:
    if omega < 0.0:
        raise ValueError("omega must be >= 0")
    n_ao, n_aux = molecule.n_ao, molecule.n_aux
    if n_ao <= 0 or n_aux <= 0:
        raise ValueError("molecule needs orbital and auxiliary bases")
    J3c = np.zeros((n_aux, n_ao, n_ao), dtype=np.float64, order="C")
    L = lib()
    for (li, lj), p in pair_data.items():
        P, A, B = as_f64(p.P_p, (4,)), as_f64(p.A_a, (4,)), as_f64(p.B_b, (4,))
        c, ia, ja = as_f64(p.coefficient), as_i32(p.i_ao_start), as_i32(p.j_ao_start)
        n_pair = P.shape[0]
        if n_pair == 0:
            continue
        for lk, a in auxiliary_pair_data.items():
            C, cc, ka = as_f64(a.A_a, (4,)), as_f64(a.coefficient), as_i32(a.i_ao_start)
            if C.shape[0] == 0:
                continue
            rc = L.three_center(int(li), int(lj), int(lk), dp(P), dp(A), dp(B), dp(c), ip(ia), ip(ja), n_pair,
                                dp(C), dp(cc), ip(ka), C.shape[0], dp(J3c), n_ao, n_aux,
                                bool(molecule.spherical_basis), float(omega))
            check(rc, f"three_center({li},{lj}|{lk})")
    return J3c
