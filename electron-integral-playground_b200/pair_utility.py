"""Primitive shell-pair screening and the structure-of-arrays pair tables.

These tables are the input format of the integral C ABI.  The screening rule,
its quirks and the resulting order are those of the reference front end
(electron_integral_playground/pair_utility.py:6-229):

* bound = 2 |c_a c_b| (L_i/2ea)^(L_i/2) (L_j/2eb)^(L_j/2)
          * exp(-ab/p d^2) * max((pi/p)^1.5, 2^0.25 (pi/p)^1.25),
  where d starts at |AB| and is decremented *cumulatively* by
  sqrt(L_i/2a) per bra primitive and sqrt(L_j/2b) per ket primitive, clamped
  at zero after every ket primitive (pair_utility.py:97-116);
* pairs with bound >= 1e-14 are kept (``form_pair_data`` ignores its own
  threshold argument, pair_utility.py:185-188);
* within an (l_i, l_j) class, pairs are stably sorted by descending bound.

The reference loops over shells and primitives in Python; here the same
sequence of floating-point operations runs vectorised over all shell pairs of
a class, so the pair sets, their order and the table values agree with the
reference bit for bit (checked in tests/test_pair_utility.py).
"""

import numpy as np

from .data_structure import Molecule, PrimitivePairData

REFERENCE_PAIR_THRESHOLD = 1e-14


def _shell_arrays(shells):
    n = len(shells)
    ang = np.array([s.angular for s in shells], dtype=np.int64)
    atom = np.array([s.i_atom for s in shells], dtype=np.int64)
    ao = np.array([s.i_ao_start for s in shells], dtype=np.int64)
    nprim = np.array([len(s.primitive_exponents) for s in shells], dtype=np.int64)
    kmax = int(nprim.max())
    exps = np.ones((n, kmax))
    coefs = np.zeros((n, kmax))
    for i, s in enumerate(shells):
        exps[i, : nprim[i]] = s.primitive_exponents
        coefs[i, : nprim[i]] = s.primitive_coefficients
    return ang, atom, ao, nprim, exps, coefs


def form_primitive_pair_list(molecule: Molecule, schwarz_upper_bound: float, j_shift=None):
    """Return {(l_i, l_j): (i_shell, j_shell, i_prim, j_prim, bound) arrays}, sorted.

    j_shift (not in the reference; periodic images): a 3-vector in Bohr added
    to the position of every j shell, so the pairs are (shell i in the home
    cell, shell j in the image cell at j_shift), screened by the same rule."""
    shells = molecule.basis_shells
    if not shells or molecule.n_ao <= 0:
        raise ValueError("molecule has no orbital basis attached")
    ang, atom, ao, nprim, exps, coefs = _shell_arrays(shells)
    geom = np.asarray(molecule.geometry, dtype=np.float64)
    geom_j = geom if j_shift is None else geom + np.asarray(j_shift, dtype=np.float64)[None, :]
    n = len(shells)
    # Per-primitive factors, as the reference forms them inside its loops.
    lf = ang[:, None].astype(np.float64)
    scaled = np.abs(coefs)
    with np.errstate(divide="ignore", invalid="ignore"):
        powf = np.power(lf / (2.0 * np.e * exps), lf / 2.0)
        shift = np.sqrt(lf / 2.0 / exps)
    scaled = np.where(lf > 0, scaled * powf, scaled)

    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    ii, jj = ii.ravel(), jj.ravel()  # reference loop order: i_shell outer, j_shell inner
    keep = (ang[ii] < ang[jj]) | ((ang[ii] == ang[jj]) & (ao[ii] <= ao[jj]))
    ii, jj = ii[keep], jj[keep]
    d0 = np.array([np.linalg.norm(geom[atom[a]] - geom_j[atom[b]]) for a, b in
                   zip(ii, jj)]) if len(ii) < 64 else _norms(geom, atom, ii, jj, geom_j)

    result = {}
    for li in np.unique(ang):
        for lj in np.unique(ang):
            if li > lj:
                continue
            sel = (ang[ii] == li) & (ang[jj] == lj)
            if not sel.any():
                continue
            si, sj, d = ii[sel], jj[sel], d0[sel].copy()
            npi, npj = nprim[si], nprim[sj]
            rec_ip, rec_jp, rec_bound, rec_sp = [], [], [], []
            for ip in range(int(npi.max())):
                vi = ip < npi
                d = np.where(vi, d - shift[si, ip], d)
                a = exps[si, ip]
                ca = scaled[si, ip]
                for jp in range(int(npj.max())):
                    v = vi & (jp < npj)
                    d = np.where(v, d - shift[sj, jp], d)
                    d = np.where(v, np.maximum(d, 0.0), d)
                    b = exps[sj, jp]
                    cb = scaled[sj, jp]
                    gauss = np.exp(-a * b / (a + b) * d * d)
                    cab = 2.0 * ca * cb
                    ovl = np.power(np.pi / (a + b), 1.5)
                    sch = np.power(np.pi / (a + b), 1.25) * np.power(2, 0.25)
                    bound = cab * gauss * np.maximum(ovl, sch)
                    ok = v & ~(bound < schwarz_upper_bound)
                    idx = np.nonzero(ok)[0]
                    rec_sp.append(idx)
                    rec_ip.append(np.full(idx.shape, ip))
                    rec_jp.append(np.full(idx.shape, jp))
                    rec_bound.append(bound[idx])
            sp = np.concatenate(rec_sp)
            if sp.size == 0:
                continue
            ipa, jpa, bnd = np.concatenate(rec_ip), np.concatenate(rec_jp), np.concatenate(rec_bound)
            # Reference insertion order is (shell pair, i_prim, j_prim); then a
            # stable sort by descending bound.
            order = np.lexsort((jpa, ipa, sp))
            sp, ipa, jpa, bnd = sp[order], ipa[order], jpa[order], bnd[order]
            order = np.argsort(-bnd, kind="stable")
            result[(int(li), int(lj))] = (si[sp[order]], sj[sp[order]], ipa[order], jpa[order], bnd[order])
    return result


def _norms(geom, atom, ii, jj, geom_j=None):
    # np.linalg.norm of a 3-vector is sqrt(dot(v, v)); evaluate it the same way
    # per unique atom pair (few), then gather.
    geom_j = geom if geom_j is None else geom_j
    na = geom.shape[0]
    key = atom[ii] * na + atom[jj]
    uk, inv = np.unique(key, return_inverse=True)
    vals = np.array([np.linalg.norm(geom[k // na] - geom_j[k % na]) for k in uk])
    return vals[inv]


def form_primitive_pair_data(molecule: Molecule, pair_list, j_shift=None) -> dict:
    """Pack a pair list into the (n, 4) [x, y, z, exponent] SoA tables the C ABI reads
    (j_shift: the image offset the list was formed with, see form_primitive_pair_list)."""
    shells = molecule.basis_shells
    ang, atom, ao, nprim, exps, coefs = _shell_arrays(shells)
    geom = np.asarray(molecule.geometry, dtype=np.float64)
    geom_j = geom if j_shift is None else geom + np.asarray(j_shift, dtype=np.float64)[None, :]
    out = {}
    for key, (si, sj, ip, jp, bnd) in pair_list.items():
        n_pair = si.shape[0]
        A = geom[atom[si]]
        B = geom_j[atom[sj]]
        a = exps[si, ip]
        b = exps[sj, jp]
        p = a + b
        P = (a[:, None] * A + b[:, None] * B) / p[:, None]
        dAB = A - B
        d2 = _row_dot(dAB)
        gauss = np.exp(-a * b / p * d2)
        coef = coefs[si, ip] * coefs[sj, jp] * gauss
        data = PrimitivePairData(
            P_p=np.ascontiguousarray(np.concatenate([P, p[:, None]], axis=1)),
            A_a=np.ascontiguousarray(np.concatenate([A, a[:, None]], axis=1)),
            B_b=np.ascontiguousarray(np.concatenate([B, b[:, None]], axis=1)),
            coefficient=np.ascontiguousarray(coef),
            i_ao_start=ao[si].astype(np.int32),
            j_ao_start=ao[sj].astype(np.int32),
            i_atom=atom[si].astype(np.int32),
            j_atom=atom[sj].astype(np.int32),
            upper_bound=np.ascontiguousarray(bnd),
        )
        assert data.P_p.shape == (n_pair, 4)
        out[key] = data
    return out


def _row_dot(v):
    # (A - B) @ (A - B) per row; the stacked matmul evaluates each 3-term inner
    # product with the same kernel as numpy's 1-D dot (bit-identical).
    return np.matmul(v[:, None, :], v[:, :, None])[:, 0, 0]


def form_pair_data(molecule: Molecule, schwarz_upper_bound: float) -> dict:
    """Orbital pair tables; like the reference, the screening threshold is fixed at 1e-14."""
    return form_primitive_pair_data(molecule, form_primitive_pair_list(molecule, REFERENCE_PAIR_THRESHOLD))


def form_primitive_auxiliary_pair_data(molecule: Molecule) -> dict:
    shells = molecule.auxiliary_basis_shells
    if not shells or molecule.n_aux <= 0:
        raise ValueError("molecule has no auxiliary basis attached")
    geom = np.asarray(molecule.geometry, dtype=np.float64)
    out = {}
    for l in sorted({s.angular for s in shells}):
        group = [s for s in shells if s.angular == l]
        rows, coef, start, at = [], [], [], []
        for s in group:
            for e, c in zip(s.primitive_exponents, s.primitive_coefficients):
                rows.append([*geom[s.i_atom], e])
                coef.append(c)
                start.append(s.i_ao_start)
                at.append(s.i_atom)
        out[l] = PrimitivePairData(
            P_p=None, A_a=np.ascontiguousarray(np.array(rows, dtype=np.float64).reshape(-1, 4)),
            B_b=None, coefficient=np.array(coef, dtype=np.float64),
            i_ao_start=np.array(start, dtype=np.int32), j_ao_start=None,
            i_atom=np.array(at, dtype=np.int32), j_atom=None)
    return out


def form_auxiliary_pair_data(molecule: Molecule) -> dict:
    return form_primitive_auxiliary_pair_data(molecule)
