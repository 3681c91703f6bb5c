"""Generate csrc/generated/sph_tables.h: Cartesian -> real-solid-harmonic coefficients.

For angular momentum l the table row m (order S_{l,l}..S_{l,1}, C_{l,0}..C_{l,l})
holds the coefficient of x^a y^b z^c (Cartesian order: a from l down to 0,
then b from l-a down to 0) in

    C_{l,m} = sqrt((2 - delta_m0) (l-m)!/(l+m)!) Pi_{l,m}(z, r) A_m(x, y)
    S_{l,m} = sqrt(2 (l-m)!/(l+m)!)              Pi_{l,m}(z, r) B_m(x, y)
    Pi_{l,m} = sum_k (-1)^k 2^-l C(l,k) C(2l-2k,l) (l-2k)!/(l-2k-m)! r^2k z^(l-2k-m)
    A_m = sum_p C(m,p) x^p y^(m-p) cos(pi (m-p)/2),  B_m = ... sin(pi (m-p)/2)

(the definitions documented in the reference,
c_library/cartesian_spherical_transformation.hpp:7-17).  Applied to raw
Cartesian integrals of shells normalised on their pure-x component, these rows
give the spherical integrals directly (the per-component Cartesian
normalisation of the reference cancels against its anti-normalised table).
l = 0 and l = 1 are identities (p stays x, y, z, as in the reference).

Also emits the per-component Cartesian normalisation
sqrt((2l)!/l! * a!b!c!/((2a)!(2b)!(2c)!)) used for Cartesian output.

Exact rational arithmetic, square roots in 40-digit decimal; run
``python gen_tables.py`` after changing it (the header is committed).
"""

import decimal
import pathlib
from fractions import Fraction
from math import comb, factorial

LMAX = 9
decimal.getcontext().prec = 40


def cart(l):
    return [(a, b, l - a - b) for a in range(l, -1, -1) for b in range(l - a, -1, -1)]


def poly_mul(p, q):
    out = {}
    for k1, v1 in p.items():
        for k2, v2 in q.items():
            k = (k1[0] + k2[0], k1[1] + k2[1], k1[2] + k2[2])
            out[k] = out.get(k, Fraction(0)) + v1 * v2
    return out


def solid_harmonic_rows(l):
    """Rows as (rational polynomial coefficients, norm^2 rational)."""
    rows = []
    for kind, ms in (("S", range(l, 0, -1)), ("C", range(0, l + 1))):
        for m in ms:
            pi = {}
            for k in range((l - m) // 2 + 1):
                g = Fraction((-1) ** k * comb(l, k) * comb(2 * l - 2 * k, l) * factorial(l - 2 * k),
                             factorial(l - 2 * k - m) * 2 ** l)
                for a in range(k + 1):
                    for b in range(k - a + 1):
                        c = k - a - b
                        mult = factorial(k) // (factorial(a) * factorial(b) * factorial(c))
                        key = (2 * a, 2 * b, 2 * c + l - 2 * k - m)
                        pi[key] = pi.get(key, Fraction(0)) + g * mult
            ab = {}
            for p in range(m + 1):
                r4 = (m - p) % 4
                trig = ({1: 1, 3: -1}.get(r4, 0) if kind == "S" else {0: 1, 2: -1}.get(r4, 0))
                if trig:
                    ab[(p, m - p, 0)] = ab.get((p, m - p, 0), Fraction(0)) + comb(m, p) * trig
            norm2 = Fraction((2 if (kind == "S" or m > 0) else 1) * factorial(l - m), factorial(l + m))
            rows.append((poly_mul(pi, ab), norm2))
    return rows


def dec_sqrt(fr):
    return (decimal.Decimal(fr.numerator) / decimal.Decimal(fr.denominator)).sqrt()


def fmt(x):
    v = float(x)
    return "0.0" if v == 0.0 else repr(v)


def main():
    lines = ["// Generated by gen_tables.py -- do not edit.", "#pragma once", "",
             f"#define EIP_SPH_LMAX {LMAX}", ""]
    offsets, flat = [], []
    for l in range(LMAX + 1):
        nc = (l + 1) * (l + 2) // 2
        offsets.append(len(flat))
        if l <= 1:
            for i in range(nc):
                flat.extend(1.0 if i == j else 0.0 for j in range(nc))
            continue
        for poly, norm2 in solid_harmonic_rows(l):
            s = dec_sqrt(norm2)
            for comp in cart(l):
                flat.append(decimal.Decimal(poly.get(comp, Fraction(0)).numerator) /
                            decimal.Decimal(poly.get(comp, Fraction(0)).denominator) * s)
    lines.append("// Row-major (2l+1) x (l+1)(l+2)/2 blocks, l = 0..EIP_SPH_LMAX.")
    lines.append("constexpr int eip_sph_offset[EIP_SPH_LMAX + 2] = {"
                 + ", ".join(str(o) for o in offsets + [len(flat)]) + "};")
    lines.append(f"constexpr double eip_sph_coef[{len(flat)}] = {{")
    for i in range(0, len(flat), 6):
        lines.append("    " + ", ".join(fmt(v) for v in flat[i:i + 6]) + ",")
    lines.append("};")
    lines.append("")
    norms, noff = [], []
    for l in range(LMAX + 1):
        noff.append(len(norms))
        for (a, b, c) in cart(l):
            fr = Fraction(factorial(2 * l) * factorial(a) * factorial(b) * factorial(c),
                          factorial(l) * factorial(2 * a) * factorial(2 * b) * factorial(2 * c))
            norms.append(dec_sqrt(fr))
    lines.append("constexpr int eip_cart_norm_offset[EIP_SPH_LMAX + 2] = {"
                 + ", ".join(str(o) for o in noff + [len(norms)]) + "};")
    lines.append(f"constexpr double eip_cart_norm[{len(norms)}] = {{")
    for i in range(0, len(norms), 6):
        lines.append("    " + ", ".join(fmt(v) for v in norms[i:i + 6]) + ",")
    lines.append("};")
    out = pathlib.Path(__file__).resolve().parent / "generated" / "sph_tables.h"
    out.parent.mkdir(exist_ok=True)
    out.write_text("\n".join(lines) + "\n")
    print("wrote", out, len(flat), "coefficients")


if __name__ == "__main__":
    main()
