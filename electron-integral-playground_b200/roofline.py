"""Algorithmic work of the (mu nu|P) path, used by bench.py for rooflines.

Per primitive triplet of class (a, b | c), L = a + b + c, the algorithmic
FLOP count is

  W(a,b,c) = 2 H(a+b) sum_{k in cart(c)} prod_d (floor(k_d/2)+1)        ket stage
           + 2 ncart(c) sum_{i in cart(a), j in cart(b)} prod_d (i_d+j_d+1)  bra stage
           + 2 N_R(L) + 20 (L+1)                                       R tetrahedron + Boys
  H(n) = C(n+3, 3),  N_R(L) = sum_{t+u+v<=L} prod (floor(t/2)+1)(floor(u/2)+1)(floor(v/2)+1)

and the algorithmic bytes are the packed output (8 bytes per spherical
element, each contracted block written once) plus the input tables.

Units of work: primitive triplets (n_pair x n_aux_primitive per class, the
reference's loop, MI/three_center.cpp:309-316) and contracted shell triplets;
"screened" triplets are the contracted ones whose bound Q_pair * Q_aux is at
least the threshold, with
  Q_pair = sum over the shell pair's primitive pairs of the front end's pair
           bound (pair_utility.py:97-116: an upper bound of sqrt((ab|ab)) and of
           the overlap), and
  Q_aux  = sum_k |c_k| 2 (l/(2 e q_k))^(l/2) sqrt(2 pi^(5/2) / (q_k^2 sqrt(2 q_k))),
           the same construction applied to one auxiliary function.
"""

from math import comb, e, pi, sqrt

import numpy as np


def cart(l):
    return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]


def n_r(L):
    return sum((t // 2 + 1) * (u // 2 + 1) * (v // 2 + 1)
               for t in range(L + 1) for u in range(L + 1 - t) for v in range(L + 1 - t - u))


def flops_per_primitive_triplet(a, b, c):
    L = a + b + c
    ket = 2 * comb(a + b + 3, 3) * sum((k[0] // 2 + 1) * (k[1] // 2 + 1) * (k[2] // 2 + 1) for k in cart(c))
    bra = 2 * len(cart(c)) * sum((i[0] + j[0] + 1) * (i[1] + j[1] + 1) * (i[2] + j[2] + 1)
                                 for i in cart(a) for j in cart(b))
    return ket + bra + 2 * n_r(L) + 20 * (L + 1)


def _q_aux(l, q, c):
    f = np.power(l / (2.0 * e * q), l / 2.0) if l > 0 else np.ones_like(q)
    return np.abs(c) * 2.0 * f * np.sqrt(2.0 * pi ** 2.5 / (q * q * np.sqrt(2.0 * q)))


def class_statistics(pair_data, aux_data, threshold=1e-14, spherical=True):
    """Per (l_i, l_j, l_k) class: primitive triplets, contracted triplets,
    screened triplets, algorithmic FLOPs and output bytes."""
    out = {}
    n_of = (lambda l: 2 * l + 1) if spherical else (lambda l: (l + 1) * (l + 2) // 2)
    aux_q = {}
    for lk, a in aux_data.items():
        starts = np.asarray(a.i_ao_start)
        qk = _q_aux(lk, a.A_a[:, 3], np.asarray(a.coefficient))
        u, inv = np.unique(starts, return_inverse=True)
        aux_q[lk] = (np.bincount(inv, weights=qk), a.A_a.shape[0])
    for (li, lj), p in pair_data.items():
        key = np.asarray(p.i_ao_start).astype(np.int64) * (1 << 32) + np.asarray(p.j_ao_start)
        u, inv = np.unique(key, return_inverse=True)
        bnd = p.upper_bound if getattr(p, "upper_bound", None) is not None else np.ones(key.shape[0])
        q_pair = np.bincount(inv, weights=bnd)
        n_pp = p.P_p.shape[0]
        for lk, (q_aux, n_auxprim) in aux_q.items():
            n_sp, n_ax = q_pair.shape[0], q_aux.shape[0]
            qa = np.sort(q_aux)
            # number of (pair, aux) with q_pair * q_aux >= threshold
            screened = int(np.sum(n_ax - np.searchsorted(qa, threshold / np.maximum(q_pair, 1e-300), side="left")))
            prim = n_pp * n_auxprim
            out[(li, lj, lk)] = dict(
                primitive=prim, contracted=n_sp * n_ax, screened=screened,
                flops=prim * flops_per_primitive_triplet(li, lj, lk),
                out_bytes=8 * n_sp * n_ax * n_of(li) * n_of(lj) * n_of(lk),
                in_bytes=112 * n_pp + 44 * n_auxprim)
    return out


def totals(stats_list):
    keys = ("primitive", "contracted", "screened", "flops", "out_bytes", "in_bytes")
    tot = {k: 0 for k in keys}
    per_class = {}
    for st in stats_list:
        for cls, d in st.items():
            pc = per_class.setdefault(cls, {k: 0 for k in keys})
            for k in keys:
                tot[k] += d[k]
                pc[k] += d[k]
    return tot, per_class
