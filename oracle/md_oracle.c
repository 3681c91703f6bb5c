/*
 * CPU oracle for the McMurchie-Davidson integral path -- TEST INFRASTRUCTURE.
 * Used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * as the reference to verify against; never linked into, or called by, the product library.
 *
 * Restatement of the reference drivers, primitive triplet by primitive
 * triplet, in plain C with runtime angular momenta:
 *   three_center       MI/three_center.cpp:27-173 (kernel), :175-289 (scatter)
 *   two_center         MI/two_center.cpp:25-120, :122-212 (lower-triangle skip :138)
 *   nuclear_attraction MI/nuclear_attraction.cpp:23-114, :116-171
 *   overlap            MI/overlap.cpp:16-79, :81-128
 * (MI/ = electron_integral_playground/c_library/molecular_integral/.)
 * Building blocks follow the mathematics the reference documents:
 *   E^{i,0}_t vertical recursion      c_library/mcmurchie_davidson_E_term.hpp:7-45
 *   E^{i,j}_t binomial transfer       c_library/mcmurchie_davidson_E_term.hpp:158-199
 *   one-centre (auxiliary) E          c_library/mcmurchie_davidson_E_term.hpp:96-130
 *   R^n_{tuv}, R^n_000 = (-2z)^n F_n  c_library/mcmurchie_davidson_R_term.hpp:9-28
 *   Cartesian normalisation           c_library/kernel_cartesian_normalization.hpp:22-26
 *   real solid harmonics, order       c_library/cartesian_spherical_transformation.hpp:7-17,38-39
 * The R tetrahedron is built with the Hermite recursion
 *   R^n_{t+1,u,v} = t R^{n+1}_{t-1,u,v} + X_PC R^{n+1}_{t,u,v}
 * (same values as the reference's closed form).  The Boys function is NOT the
 * reference's Chebyshev table: it is the convergent series
 *   F_m(T) = e^{-T} sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1))
 * in long double (T <= 60), else erf + upward recursion, so that the oracle
 * is accurate to rounding; the reference's table is accurate to ~5e-14
 * relative (boys_function.hpp:71).
 */
#include "md_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OR_MAX_ORB 6
#define OR_MAX_AUX 9
#define OR_MAX_CART 55 /* (9+1)(9+2)/2 */

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

/* Cartesian component c of angular momentum l in the reference order
 * (x from l down to 0, then y from l-x down to 0; indexing.hpp:97-115). */
static void cart_comp(int l, int c, int* x, int* y, int* z) {
    int idx = 0;
    for (int a = l; a >= 0; a--)
        for (int b = l - a; b >= 0; b--) {
            if (idx == c) { *x = a; *y = b; *z = l - a - b; return; }
            idx++;
        }
}

void oracle_boys(int L, double xd, double* y) {
    long double T = xd;
    if (T < 1e-300L) {
        for (int m = 0; m <= L; m++) y[m] = 1.0 / (2 * m + 1);
        return;
    }
    long double eT = expl(-T);
    long double F[64];
    if (T <= 60.0L) {
        long double term = 1.0L / (2 * L + 1), sum = term;
        for (int k = 1; k < 4000; k++) {
            term *= 2.0L * T / (2 * L + 2 * k + 1);
            sum += term;
            if (term < sum * 1e-22L) break;
        }
        F[L] = eT * sum;
        for (int m = L - 1; m >= 0; m--) F[m] = (2.0L * T * F[m + 1] + eT) / (2 * m + 1);
    } else {
        long double sT = sqrtl(T);
        F[0] = 0.5L * sqrtl(3.14159265358979323846264338327950288L) * erfl(sT) / sT;
        for (int m = 0; m < L; m++) F[m + 1] = ((2 * m + 1) * F[m] - eT) / (2.0L * T);
    }
    for (int m = 0; m <= L; m++) y[m] = (double)F[m];
}

/* F_m(x[i]), m = 0..L, for n arguments: y[i * (L + 1) + m]. */
void oracle_boys_many(int L, int n, const double* x, double* y) {
    for (int i = 0; i < n; i++) oracle_boys(L, x[i], y + (size_t)i * (L + 1));
}

/* ---- real solid harmonics as polynomials in x, y, z --------------------- */
typedef struct { long double c[10][10][10]; } poly3;

static long double lfact(int n) { long double r = 1; for (int i = 2; i <= n; i++) r *= i; return r; }
static long double lbinom(int n, int k) { return (k < 0 || k > n) ? 0 : lfact(n) / (lfact(k) * lfact(n - k)); }

static void poly_mul(const poly3* a, const poly3* b, poly3* out, int deg) {
    poly3 r; memset(&r, 0, sizeof r);
    for (int i = 0; i <= deg; i++) for (int j = 0; i + j <= deg; j++) for (int k = 0; i + j + k <= deg; k++) {
        long double av = a->c[i][j][k];
        if (av == 0) continue;
        for (int p = 0; i + p <= deg; p++) for (int q = 0; i + p + j + q <= deg; q++)
            for (int s = 0; i + p + j + q + k + s <= deg; s++)
                r.c[i + p][j + q][k + s] += av * b->c[p][q][s];
    }
    *out = r;
}

void oracle_spherical_matrix(int l, double* out) {
    int nc = ncart(l), ns = 2 * l + 1;
    memset(out, 0, sizeof(double) * nc * ns);
    if (l <= 1) { /* s, and p kept as (x, y, z) */
        for (int i = 0; i < nc; i++) out[i * nc + i] = 1.0;
        return;
    }
    int row = 0;
    for (int pass = 0; pass < 2; pass++) {
        int m_begin = pass == 0 ? l : 0, m_end = pass == 0 ? 0 : l + 1, step = pass == 0 ? -1 : 1;
        for (int m = m_begin; m != m_end; m += step) {
            /* Pi_{l,m}(z, r) = sum_k gamma_{l,k,m} r^{2k} z^{l-2k-m} */
            poly3 pi; memset(&pi, 0, sizeof pi);
            for (int k = 0; k <= (l - m) / 2; k++) {
                long double g = ((k % 2) ? -1.0L : 1.0L) * lbinom(l, k) * lbinom(2 * l - 2 * k, l) *
                                lfact(l - 2 * k) / lfact(l - 2 * k - m) / powl(2.0L, l);
                /* r^{2k} = (x^2+y^2+z^2)^k, multinomial */
                for (int a = 0; a <= k; a++) for (int b = 0; a + b <= k; b++) {
                    int c = k - a - b;
                    long double mult = lfact(k) / (lfact(a) * lfact(b) * lfact(c));
                    pi.c[2 * a][2 * b][2 * c + l - 2 * k - m] += g * mult;
                }
            }
            poly3 ab; memset(&ab, 0, sizeof ab);
            for (int p = 0; p <= m; p++) {
                int r4 = (m - p) % 4;
                long double trig = pass == 0 ? (r4 == 1 ? 1.0L : (r4 == 3 ? -1.0L : 0.0L))
                                             : (r4 == 0 ? 1.0L : (r4 == 2 ? -1.0L : 0.0L));
                ab.c[p][m - p][0] += lbinom(m, p) * trig;
            }
            long double norm = sqrtl((pass == 0 || m > 0 ? 2.0L : 1.0L) * lfact(l - m) / lfact(l + m));
            poly3 prod; poly_mul(&pi, &ab, &prod, l);
            for (int c = 0; c < nc; c++) {
                int x, y, z; cart_comp(l, c, &x, &y, &z);
                out[row * nc + c] = (double)(norm * prod.c[x][y][z]);
            }
            row++;
        }
    }
}

/* sqrt((2L)!/L! * x!y!z!/((2x)!(2y)!(2z)!)), kernel_cartesian_normalization.hpp:22-26 */
static double cart_norm(int l, int c) {
    int x, y, z; cart_comp(l, c, &x, &y, &z);
    long double v = lfact(2 * l) / lfact(l) * lfact(x) * lfact(y) * lfact(z) /
                    (lfact(2 * x) * lfact(2 * y) * lfact(2 * z));
    return (double)sqrtl(v);
}

/* E^{i,0}_t for i <= n (vertical recursion), E[i*(n+1)+t]. */
static void e_vertical(int n, double PA, double inv2p, double* E) {
    memset(E, 0, sizeof(double) * (n + 1) * (n + 1));
    E[0] = 1.0;
    for (int i = 0; i < n; i++)
        for (int t = 0; t <= i + 1; t++) {
            double v = 0.0;
            if (t >= 1) v += inv2p * E[i * (n + 1) + t - 1];
            if (t <= i) v += PA * E[i * (n + 1) + t];
            if (t + 1 <= i) v += (t + 1) * E[i * (n + 1) + t + 1];
            E[(i + 1) * (n + 1) + t] = v;
        }
}

/* E^{i,j}_t = sum_m binom(j, j-m) AB^{j-m} E^{i+m,0}_t, stored [i][j][t] with t <= i+j. */
static void e_pair(int li, int lj, double PA, double AB, double inv2p, double* Eij) {
    int n = li + lj;
    double Ev[(2 * OR_MAX_AUX + 1) * (2 * OR_MAX_AUX + 1)];
    e_vertical(n, PA, inv2p, Ev);
    for (int i = 0; i <= li; i++)
        for (int j = 0; j <= lj; j++)
            for (int t = 0; t <= n; t++) {
                double v = 0.0;
                if (t <= i + j) {
                    double abp = 1.0;
                    for (int m = j; m >= 0; m--) {
                        if (t <= i + m) v += lbinom(j, j - m) * abp * Ev[(i + m) * (n + 1) + t];
                        abp *= AB;
                    }
                }
                Eij[(i * (lj + 1) + j) * (n + 1) + t] = v;
            }
}

/* R^0_{tuv} for t+u+v <= L into R0[(t*(L+1)+u)*(L+1)+v]. */
static void r_tetra(int L, double zeta, double X, double Y, double Z, double* R0) {
    int S = L + 1;
    double* R = (double*)calloc((size_t)S * S * S * S, sizeof(double));
    double F[64];
    oracle_boys(L, zeta * (X * X + Y * Y + Z * Z), F);
    double f = 1.0;
    for (int n = 0; n <= L; n++) { R[(size_t)n * S * S * S] = f * F[n]; f *= -2.0 * zeta; }
#define RI(n, t, u, v) R[(((size_t)(n) * S + (t)) * S + (u)) * S + (v)]
    for (int N = 1; N <= L; N++)
        for (int t = 0; t <= N; t++)
            for (int u = 0; t + u <= N; u++) {
                int v = N - t - u;
                for (int n = 0; n + N <= L; n++) {
                    double val;
                    if (t > 0) val = (t > 1 ? (t - 1) * RI(n + 1, t - 2, u, v) : 0.0) + X * RI(n + 1, t - 1, u, v);
                    else if (u > 0) val = (u > 1 ? (u - 1) * RI(n + 1, t, u - 2, v) : 0.0) + Y * RI(n + 1, t, u - 1, v);
                    else val = (v > 1 ? (v - 1) * RI(n + 1, t, u, v - 2) : 0.0) + Z * RI(n + 1, t, u, v - 1);
                    RI(n, t, u, v) = val;
                }
            }
    for (int t = 0; t <= L; t++) for (int u = 0; t + u <= L; u++) for (int v = 0; t + u + v <= L; v++)
        R0[(t * S + u) * S + v] = RI(0, t, u, v);
#undef RI
    free(R);
}

/* raw[c] (Cartesian, pure-x normalised shells) -> spherical or normalised Cartesian block. */
static void transform_3(int li, int lj, int lk, bool spherical, const double* raw, double* out) {
    int ni = ncart(li), nj = ncart(lj), nk = ncart(lk);
    if (!spherical) {
        for (int a = 0; a < ni; a++) for (int b = 0; b < nj; b++) for (int c = 0; c < nk; c++)
            out[(a * nj + b) * nk + c] = raw[(a * nj + b) * nk + c] * cart_norm(li, a) * cart_norm(lj, b) * cart_norm(lk, c);
        return;
    }
    int si = 2 * li + 1, sj = 2 * lj + 1, sk = 2 * lk + 1;
    double *Pi = malloc(sizeof(double) * si * ni), *Pj = malloc(sizeof(double) * sj * nj), *Pk = malloc(sizeof(double) * sk * nk);
    oracle_spherical_matrix(li, Pi); oracle_spherical_matrix(lj, Pj); oracle_spherical_matrix(lk, Pk);
    double* t1 = calloc((size_t)si * nj * nk, sizeof(double));
    double* t2 = calloc((size_t)si * sj * nk, sizeof(double));
    for (int A = 0; A < si; A++) for (int a = 0; a < ni; a++) { double w = Pi[A * ni + a]; if (w == 0) continue;
        for (int bc = 0; bc < nj * nk; bc++) t1[A * nj * nk + bc] += w * raw[a * nj * nk + bc]; }
    for (int A = 0; A < si; A++) for (int B = 0; B < sj; B++) for (int b = 0; b < nj; b++) { double w = Pj[B * nj + b]; if (w == 0) continue;
        for (int c = 0; c < nk; c++) t2[(A * sj + B) * nk + c] += w * t1[(A * nj + b) * nk + c]; }
    for (int AB = 0; AB < si * sj; AB++) for (int C = 0; C < sk; C++) {
        double v = 0.0;
        for (int c = 0; c < nk; c++) v += Pk[C * nk + c] * t2[AB * nk + c];
        out[AB * sk + C] = v;
    }
    free(Pi); free(Pj); free(Pk); free(t1); free(t2);
}

static const double PI_ = 3.14159265358979323846;

int oracle_three_center(int i_L, int j_L, int k_L, const double* pair_P_p, const double* pair_A_a,
                        const double* pair_B_b, const double* pair_coefficient, const int* pair_i_ao_start,
                        const int* pair_j_ao_start, int n_pair_ij, const double* aux_A_a,
                        const double* aux_coefficient, const int* aux_i_aux_start, int n_aux_primitive_k,
                        double* J3c, int n_ao, int n_aux, bool spherical, double omega) {
    (void)n_aux;
    if (i_L < 0 || j_L < 0 || k_L < 0 || i_L > j_L || j_L > OR_MAX_ORB || k_L > OR_MAX_AUX) {
        printf("%s does not support angular i_L = %d, j_L = %d, k_L = %d\n", __func__, i_L, j_L, k_L);
        fflush(stdout);
        return 1;
    }
    int L = i_L + j_L + k_L, S = L + 1, nij = i_L + j_L + 1;
    int ni = ncart(i_L), nj = ncart(j_L), nk = ncart(k_L);
    int oi = spherical ? 2 * i_L + 1 : ni, oj = spherical ? 2 * j_L + 1 : nj, ok = spherical ? 2 * k_L + 1 : nk;
    double* R0 = malloc(sizeof(double) * S * S * S);
    double* raw = malloc(sizeof(double) * ni * nj * nk);
    double* blk = malloc(sizeof(double) * ni * nj * nk);
    double Ex[(OR_MAX_ORB + 1) * (OR_MAX_ORB + 1) * (2 * OR_MAX_ORB + 1)];
    double Ey[sizeof Ex / sizeof Ex[0]], Ez[sizeof Ex / sizeof Ex[0]];
    double Ek[(OR_MAX_AUX + 1) * (OR_MAX_AUX + 1)];
    for (int ip = 0; ip < n_pair_ij; ip++) {
        const double* P = pair_P_p + 4 * ip; const double* A = pair_A_a + 4 * ip; const double* B = pair_B_b + 4 * ip;
        double p = P[3];
        e_pair(i_L, j_L, P[0] - A[0], A[0] - B[0], 0.5 / p, Ex);
        e_pair(i_L, j_L, P[1] - A[1], A[1] - B[1], 0.5 / p, Ey);
        e_pair(i_L, j_L, P[2] - A[2], A[2] - B[2], 0.5 / p, Ez);
        for (int ia = 0; ia < n_aux_primitive_k; ia++) {
            const double* C = aux_A_a + 4 * ia;
            double q = C[3];
            double coef = pair_coefficient[ip] * aux_coefficient[ia];
            double pref, zeta;
            if (omega == 0.0) { pref = coef * 2.0 * pow(PI_, 2.5) / (p * q * sqrt(p + q)); zeta = p * q / (p + q); }
            else { pref = coef * 2.0 * pow(PI_, 2.5) * omega / (p * q * sqrt(p * q + (p + q) * omega * omega));
                   zeta = 1.0 / (1.0 / p + 1.0 / q + 1.0 / (omega * omega)); }
            e_vertical(k_L, 0.0, 0.5 / q, Ek);
            r_tetra(L, zeta, P[0] - C[0], P[1] - C[1], P[2] - C[2], R0);
            for (int a = 0; a < ni; a++) { int ix, iy, iz; cart_comp(i_L, a, &ix, &iy, &iz);
            for (int b = 0; b < nj; b++) { int jx, jy, jz; cart_comp(j_L, b, &jx, &jy, &jz);
            for (int c = 0; c < nk; c++) { int kx, ky, kz; cart_comp(k_L, c, &kx, &ky, &kz);
                double v = 0.0;
                for (int t = 0; t <= ix + jx; t++) { double ex = Ex[(ix * (j_L + 1) + jx) * nij + t];
                for (int u = 0; u <= iy + jy; u++) { double ey = Ey[(iy * (j_L + 1) + jy) * nij + u];
                for (int w = 0; w <= iz + jz; w++) { double ez = Ez[(iz * (j_L + 1) + jz) * nij + w];
                    double e = ex * ey * ez;
                    for (int sx = kx % 2; sx <= kx; sx += 2) for (int sy = ky % 2; sy <= ky; sy += 2)
                    for (int sz = kz % 2; sz <= kz; sz += 2) {
                        double ek = Ek[kx * (k_L + 1) + sx] * Ek[ky * (k_L + 1) + sy] * Ek[kz * (k_L + 1) + sz];
                        double sign = ((sx + sy + sz) % 2) ? -1.0 : 1.0;
                        v += sign * e * ek * R0[((t + sx) * S + (u + sy)) * S + (w + sz)];
                    } } } }
                raw[(a * nj + b) * nk + c] = pref * v;
            } } }
            transform_3(i_L, j_L, k_L, spherical, raw, blk);
            long ia0 = pair_i_ao_start[ip], ja0 = pair_j_ao_start[ip], ka0 = aux_i_aux_start[ia];
            long nao = n_ao;
            for (int a = 0; a < oi; a++) for (int b = 0; b < oj; b++) for (int c = 0; c < ok; c++) {
                double v = blk[(a * oj + b) * ok + c];
                J3c[(ka0 + c) * nao * nao + (ia0 + a) * nao + (ja0 + b)] += v;
                if (ia0 != ja0) J3c[(ka0 + c) * nao * nao + (ja0 + b) * nao + (ia0 + a)] += v;
            }
        }
    }
    free(R0); free(raw); free(blk);
    return 0;
}

/* Two one-centre Hermite expansions; (-1)^|s| on the ket. */
int oracle_two_center(int i_L, int j_L, const double* aux_A_a, const double* aux_i_coefficient,
                      const int* aux_i_aux_start, int n_aux_primitive_i, const double* aux_B_b,
                      const double* aux_j_coefficient, const int* aux_j_aux_start, int n_aux_primitive_j,
                      double* J2c, int n_aux, bool spherical, double omega) {
    if (i_L < 0 || j_L < 0 || i_L > j_L || j_L > OR_MAX_AUX) {
        printf("%s does not support angular i_L = %d, j_L = %d\n", __func__, i_L, j_L);
        fflush(stdout);
        return 1;
    }
    int L = i_L + j_L, S = L + 1, ni = ncart(i_L), nj = ncart(j_L);
    int oi = spherical ? 2 * i_L + 1 : ni, oj = spherical ? 2 * j_L + 1 : nj;
    double* R0 = malloc(sizeof(double) * S * S * S);
    double* raw = malloc(sizeof(double) * ni * nj);
    double* blk = malloc(sizeof(double) * ni * nj);
    double Ei[(OR_MAX_AUX + 1) * (OR_MAX_AUX + 1)], Ej[(OR_MAX_AUX + 1) * (OR_MAX_AUX + 1)];
    for (int ia = 0; ia < n_aux_primitive_i; ia++)
        for (int ja = 0; ja < n_aux_primitive_j; ja++) {
            long i0 = aux_i_aux_start[ia], j0 = aux_j_aux_start[ja];
            if (i_L == j_L && i0 > j0) continue;
            const double* A = aux_A_a + 4 * ia; const double* B = aux_B_b + 4 * ja;
            double p = A[3], q = B[3], coef = aux_i_coefficient[ia] * aux_j_coefficient[ja], pref, zeta;
            if (omega == 0.0) { pref = coef * 2.0 * pow(PI_, 2.5) / (p * q * sqrt(p + q)); zeta = p * q / (p + q); }
            else { pref = coef * 2.0 * pow(PI_, 2.5) * omega / (p * q * sqrt(p * q + (p + q) * omega * omega));
                   zeta = 1.0 / (1.0 / p + 1.0 / q + 1.0 / (omega * omega)); }
            e_vertical(i_L, 0.0, 0.5 / p, Ei);
            e_vertical(j_L, 0.0, 0.5 / q, Ej);
            r_tetra(L, zeta, A[0] - B[0], A[1] - B[1], A[2] - B[2], R0);
            for (int a = 0; a < ni; a++) { int ix, iy, iz; cart_comp(i_L, a, &ix, &iy, &iz);
            for (int b = 0; b < nj; b++) { int jx, jy, jz; cart_comp(j_L, b, &jx, &jy, &jz);
                double v = 0.0;
                for (int tx = ix % 2; tx <= ix; tx += 2) for (int ty = iy % 2; ty <= iy; ty += 2)
                for (int tz = iz % 2; tz <= iz; tz += 2) {
                    double e1 = Ei[ix * (i_L + 1) + tx] * Ei[iy * (i_L + 1) + ty] * Ei[iz * (i_L + 1) + tz];
                    for (int sx = jx % 2; sx <= jx; sx += 2) for (int sy = jy % 2; sy <= jy; sy += 2)
                    for (int sz = jz % 2; sz <= jz; sz += 2) {
                        double e2 = Ej[jx * (j_L + 1) + sx] * Ej[jy * (j_L + 1) + sy] * Ej[jz * (j_L + 1) + sz];
                        double sign = ((sx + sy + sz) % 2) ? -1.0 : 1.0;
                        v += sign * e1 * e2 * R0[((tx + sx) * S + (ty + sy)) * S + (tz + sz)];
                    } }
                raw[a * nj + b] = pref * v;
            } }
            transform_3(i_L, j_L, 0, spherical, raw, blk);
            long na = n_aux;
            for (int a = 0; a < oi; a++) for (int b = 0; b < oj; b++) {
                double v = blk[a * oj + b];
                J2c[(i0 + a) * na + (j0 + b)] += v;
                if (i0 != j0) J2c[(j0 + b) * na + (i0 + a)] += v;
            }
        }
    free(R0); free(raw); free(blk);
    return 0;
}

int oracle_nuclear_attraction(int i_L, int j_L, const double* pair_P_p, const double* pair_A_a,
                              const double* pair_B_b, const double* pair_coefficient, const int* pair_i_ao_start,
                              const int* pair_j_ao_start, int n_pair, const double* charge_position,
                              int n_charge, double* V, int n_ao, bool spherical, double omega) {
    if (i_L < 0 || j_L < 0 || i_L > j_L || j_L > OR_MAX_ORB) {
        printf("%s does not support angular i_L = %d, j_L = %d\n", __func__, i_L, j_L);
        fflush(stdout);
        return 1;
    }
    int L = i_L + j_L, S = L + 1, nij = L + 1, ni = ncart(i_L), nj = ncart(j_L);
    int oi = spherical ? 2 * i_L + 1 : ni, oj = spherical ? 2 * j_L + 1 : nj;
    double* R0 = malloc(sizeof(double) * S * S * S);
    double* raw = malloc(sizeof(double) * ni * nj);
    double* blk = malloc(sizeof(double) * ni * nj);
    double Ex[(OR_MAX_ORB + 1) * (OR_MAX_ORB + 1) * (2 * OR_MAX_ORB + 1)];
    double Ey[sizeof Ex / sizeof Ex[0]], Ez[sizeof Ex / sizeof Ex[0]];
    for (int ip = 0; ip < n_pair; ip++) {
        const double* P = pair_P_p + 4 * ip; const double* A = pair_A_a + 4 * ip; const double* B = pair_B_b + 4 * ip;
        double p = P[3];
        e_pair(i_L, j_L, P[0] - A[0], A[0] - B[0], 0.5 / p, Ex);
        e_pair(i_L, j_L, P[1] - A[1], A[1] - B[1], 0.5 / p, Ey);
        e_pair(i_L, j_L, P[2] - A[2], A[2] - B[2], 0.5 / p, Ez);
        double pref = (omega == 0.0) ? pair_coefficient[ip] * 2.0 * PI_ / p
                                     : pair_coefficient[ip] * 2.0 * PI_ * omega / (p * sqrt(p + omega * omega));
        double zeta = (omega == 0.0) ? p : p * omega * omega / (p + omega * omega);
        for (int ic = 0; ic < n_charge; ic++) {
            const double* C = charge_position + 3 * ic;
            r_tetra(L, zeta, P[0] - C[0], P[1] - C[1], P[2] - C[2], R0);
            for (int a = 0; a < ni; a++) { int ix, iy, iz; cart_comp(i_L, a, &ix, &iy, &iz);
            for (int b = 0; b < nj; b++) { int jx, jy, jz; cart_comp(j_L, b, &jx, &jy, &jz);
                double v = 0.0;
                for (int t = 0; t <= ix + jx; t++) for (int u = 0; u <= iy + jy; u++) for (int w = 0; w <= iz + jz; w++)
                    v += Ex[(ix * (j_L + 1) + jx) * nij + t] * Ey[(iy * (j_L + 1) + jy) * nij + u] *
                         Ez[(iz * (j_L + 1) + jz) * nij + w] * R0[(t * S + u) * S + w];
                raw[a * nj + b] = pref * v;
            } }
            transform_3(i_L, j_L, 0, spherical, raw, blk);
            long ia0 = pair_i_ao_start[ip], ja0 = pair_j_ao_start[ip], nao = n_ao, nc = n_charge;
            for (int a = 0; a < oi; a++) for (int b = 0; b < oj; b++) {
                double v = blk[a * oj + b];
                V[((ia0 + a) * nao + (ja0 + b)) * nc + ic] += v;
                if (ia0 != ja0) V[((ja0 + b) * nao + (ia0 + a)) * nc + ic] += v;
            }
        }
    }
    free(R0); free(raw); free(blk);
    return 0;
}

int oracle_overlap(int i_L, int j_L, const double* pair_A_a, const double* pair_B_b,
                   const double* pair_coefficient, const int* pair_i_ao_start, const int* pair_j_ao_start,
                   int n_pair, double* S_matrix, int n_ao, bool spherical) {
    if (i_L < 0 || j_L < 0 || i_L > j_L || j_L > OR_MAX_ORB) {
        printf("%s does not support angular i_L = %d, j_L = %d\n", __func__, i_L, j_L);
        fflush(stdout);
        return 1;
    }
    int nij = i_L + j_L + 1, ni = ncart(i_L), nj = ncart(j_L);
    int oi = spherical ? 2 * i_L + 1 : ni, oj = spherical ? 2 * j_L + 1 : nj;
    double raw[28 * 28], blk[28 * 28];
    double Ex[(OR_MAX_ORB + 1) * (OR_MAX_ORB + 1) * (2 * OR_MAX_ORB + 1)];
    double Ey[sizeof Ex / sizeof Ex[0]], Ez[sizeof Ex / sizeof Ex[0]];
    for (int ip = 0; ip < n_pair; ip++) {
        const double* A = pair_A_a + 4 * ip; const double* B = pair_B_b + 4 * ip;
        double p = A[3] + B[3], mbp = -B[3] / p;
        /* P - A = -b/p (A - B), overlap.cpp:21-28 */
        e_pair(i_L, j_L, mbp * (A[0] - B[0]), A[0] - B[0], 0.5 / p, Ex);
        e_pair(i_L, j_L, mbp * (A[1] - B[1]), A[1] - B[1], 0.5 / p, Ey);
        e_pair(i_L, j_L, mbp * (A[2] - B[2]), A[2] - B[2], 0.5 / p, Ez);
        double pref = pair_coefficient[ip] * pow(PI_ / p, 1.5);
        for (int a = 0; a < ni; a++) { int ix, iy, iz; cart_comp(i_L, a, &ix, &iy, &iz);
        for (int b = 0; b < nj; b++) { int jx, jy, jz; cart_comp(j_L, b, &jx, &jy, &jz);
            raw[a * nj + b] = pref * Ex[(ix * (j_L + 1) + jx) * nij] * Ey[(iy * (j_L + 1) + jy) * nij] *
                              Ez[(iz * (j_L + 1) + jz) * nij];
        } }
        transform_3(i_L, j_L, 0, spherical, raw, blk);
        long ia0 = pair_i_ao_start[ip], ja0 = pair_j_ao_start[ip], nao = n_ao;
        for (int a = 0; a < oi; a++) for (int b = 0; b < oj; b++) {
            double v = blk[a * oj + b];
            S_matrix[(ia0 + a) * nao + (ja0 + b)] += v;
            if (ia0 != ja0) S_matrix[(ja0 + b) * nao + (ia0 + a)] += v;
        }
    }
    return 0;
}
