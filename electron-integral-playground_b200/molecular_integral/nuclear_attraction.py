"""V[mu, nu, C] through the CUDA library; mirrors the reference nuclear_attraction.py:9-44."""

import numpy as np

from .._lib import as_f64, as_i32, check, dp, ip, lib


def nuclear_attraction(pair_data, molecule, charge_position, omega: float = 0.0) -> np.ndarray:
    if omega < 0.0:
        raise ValueError("omega must be >= 0")
    n_ao = molecule.n_ao
    if n_ao <= 0:
        raise ValueError("molecule needs an orbital basis")
    cp = np.asarray(charge_position)
    if cp.ndim != 2 or cp.shape[1] != 3 or cp.shape[0] == 0:
        raise ValueError("charge_position must be a non-empty (n, 3) array")
    cp = as_f64(cp)
    n_charge = cp.shape[0]
    V = np.zeros((n_ao, n_ao, n_charge), dtype=np.float64, order="C")
    L = lib()
    for (li, lj), p in pair_data.items():
        P, A, B = as_f64(p.P_p, (4,)), as_f64(p.A_a, (4,)), as_f64(p.B_b, (4,))
        c, ia, ja = as_f64(p.coefficient), as_i32(p.i_ao_start), as_i32(p.j_ao_start)
        if P.shape[0] == 0:
            continue
        rc = L.nuclear_attraction(int(li), int(lj), dp(P), dp(A), dp(B), dp(c), ip(ia), ip(ja), P.shape[0], dp(cp),
                                  n_charge, dp(V), n_ao, bool(molecule.spherical_basis), float(omega))
        check(rc, f"nuclear_attraction({li},{lj})")
    return V
