// Shared device-side definitions of the McMurchie-Davidson integral kernels.
//
// Index conventions (identical to the reference front end's output layout):
//   * Cartesian components of angular momentum l are ordered x-major
//     descending: for a = l..0, for b = l-a..0, c = l-a-b
//     (reference c_library/indexing.hpp:97-115).
//   * Hermite indices (t,u,v) are stored by total order N = t+u+v, and within
//     one order in the same x-major descending order, so that the tetrahedron
//     t+u+v <= L is a prefix of the one for L+1.
//   * Spherical components follow the real-solid-harmonic order
//     S_{l,l}..S_{l,1}, C_{l,0}..C_{l,l}; p stays (x, y, z)
//     (cartesian_spherical_transformation.hpp:7-17, 38-39).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

#include "generated/sph_tables.h"

namespace eip {

// ---------------------------------------------------------------- limits
constexpr int kMaxOrbitalL = 6;   // reference MAX_L (c_library/angular.h:3)
constexpr int kMaxAuxL = 9;       // reference MAX_AUX_L (c_library/angular.h:4)
constexpr int kMaxBoysM = 21;     // highest F_m any supported class needs: 6+6+9
constexpr int kBoysTaylor = 8;    // Taylor terms around each grid point
constexpr int kBoysOrders = kMaxBoysM + kBoysTaylor;  // orders tabulated: 0..28
constexpr double kBoysStep = 0.05;
constexpr double kBoysInvStep = 20.0;
constexpr int kBoysGrid = 721;    // grid points T0 = 0, 0.05, ..., 36.0
constexpr double kBoysTMax = 36.0;  // above: F_0 = sqrt(pi/T)/2 and upward recursion

// ---------------------------------------------------------------- constexpr helpers
__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int nsph(int l) { return 2 * l + 1; }
__host__ __device__ constexpr int nherm(int L) { return L < 0 ? 0 : (L + 1) * (L + 2) * (L + 3) / 6; }

__host__ __device__ constexpr int cart_x(int l, int c) {
    int idx = 0;
    for (int a = l; a >= 0; a--)
        for (int b = l - a; b >= 0; b--) {
            if (idx == c) return a;
            idx++;
        }
    return -1;
}
__host__ __device__ constexpr int cart_y(int l, int c) {
    int idx = 0;
    for (int a = l; a >= 0; a--)
        for (int b = l - a; b >= 0; b--) {
            if (idx == c) return b;
            idx++;
        }
    return -1;
}
__host__ __device__ constexpr int cart_z(int l, int c) { return l - cart_x(l, c) - cart_y(l, c); }

// Hermite index of (t,u,v) in the order-major tetrahedron.
__host__ __device__ constexpr int herm_index(int t, int u, int v) {
    int N = t + u + v;
    return nherm(N - 1) + (N - t) * (N - t + 1) / 2 + (N - t - u);
}
__host__ __device__ constexpr int herm_t(int idx) {
    int N = 0;
    while (nherm(N) <= idx) N++;
    return cart_x(N, idx - nherm(N - 1));
}
__host__ __device__ constexpr int herm_u(int idx) {
    int N = 0;
    while (nherm(N) <= idx) N++;
    return cart_y(N, idx - nherm(N - 1));
}
__host__ __device__ constexpr int herm_v(int idx) {
    int N = 0;
    while (nherm(N) <= idx) N++;
    return cart_z(N, idx - nherm(N - 1));
}

__host__ __device__ constexpr double cfact(int n) {
    double r = 1.0;
    for (int i = 2; i <= n; i++) r *= i;
    return r;
}

// One-centre Hermite coefficient of x^k exp(-q x^2):
//   E^{k,0}_s(q) = k! / (((k-s)/2)! s! 2^((k-s)/2)) * (1/(2q))^((k+s)/2)
// (closed form documented at c_library/mcmurchie_davidson_E_term.hpp:132-139);
// this returns the rational prefactor, zero when k-s is odd or s > k.
__host__ __device__ constexpr double one_centre_coef(int k, int s) {
    if (s < 0 || s > k || ((k - s) & 1)) return 0.0;
    int h = (k - s) / 2;
    double p2 = 1.0;
    for (int i = 0; i < h; i++) p2 *= 2.0;
    return cfact(k) / (cfact(h) * cfact(s) * p2);
}

// Coefficient of R^{m}_000 in the closed-form Hermite integral along one axis:
//   R_t = sum_{m=ceil(t/2)}^{t} t!/((2m-t)!(t-m)! 2^(t-m)) X^(2m-t) R^(m)
// (c_library/mcmurchie_davidson_R_term.hpp:31-37).
__host__ __device__ constexpr double hermite_r_coef(int t, int m) {
    if (m < (t + 1) / 2 || m > t) return 0.0;
    double p2 = 1.0;
    for (int i = 0; i < t - m; i++) p2 *= 2.0;
    return cfact(t) / (cfact(2 * m - t) * cfact(t - m) * p2);
}

// Real-solid-harmonic coefficient (row m, Cartesian column c) and the
// per-component Cartesian normalisation.  Only usable in constant expressions.
__host__ __device__ constexpr double sph_coef(int l, int m, int c) {
    return eip_sph_coef[eip_sph_offset[l] + m * ncart(l) + c];
}
__host__ __device__ constexpr double cart_norm_coef(int l, int c) {
    return eip_cart_norm[eip_cart_norm_offset[l] + c];
}

// Spherical-output ket coefficient of Hermite index s = (sx,sy,sz) for
// spherical component ko of a one-centre shell of angular momentum LK
// (the (1/2q) power and the (-1)^|s| sign are applied at run time).
__host__ __device__ constexpr double ket_sph_coef(int LK, int ko, int sx, int sy, int sz) {
    double r = 0.0;
    for (int c = 0; c < ncart(LK); c++) {
        double w = sph_coef(LK, ko, c);
        if (w == 0.0) continue;
        r += w * one_centre_coef(cart_x(LK, c), sx) * one_centre_coef(cart_y(LK, c), sy) *
             one_centre_coef(cart_z(LK, c), sz);
    }
    return r;
}

// Flat index of the two-centre E^{i,j}_t table along one axis,
// i <= LI, j <= LJ, t <= i+j.
template <int LJ>
__host__ __device__ constexpr int e_offset(int i, int j) {
    int o = 0;
    for (int a = 0; a < i; a++)
        for (int b = 0; b <= LJ; b++) o += a + b + 1;
    for (int b = 0; b < j; b++) o += i + b + 1;
    return o;
}
template <int LI, int LJ>
__host__ __device__ constexpr int e_size() { return e_offset<LJ>(LI + 1, 0); }

// ---------------------------------------------------------------- compile-time loops
template <int I>
using ic = std::integral_constant<int, I>;

template <int B, int E, typename F>
__device__ __forceinline__ void static_for(F&& f) {
    if constexpr (B < E) {
        f(ic<B>{});
        static_for<B + 1, E>(f);
    }
}

// ---------------------------------------------------------------- Boys function
// F_m(T) for m = 0..L, FP64.  Design (this library's own):
//   T < 36:  F_L(T) from an 8-term Taylor series around the nearest grid point
//            T0 = 0.05 i of a table of F_m(T0), m = 0..28 (built once at start-up
//            from the convergent series in long double, boys_table.cu), then the
//            stable downward recursion F_m = (2T F_{m+1} + e^-T) / (2m+1).
//   T >= 36: F_0 = sqrt(pi/T)/2 (erf(sqrt T) = 1 in FP64) and the upward
//            recursion F_{m+1} = ((2m+1) F_m - e^-T) / (2T), stable for m < T.
// `table` is the device address of the grid ((kMaxBoysM + 1) x kBoysGrid x
// kBoysTaylor doubles, order-major, see boys_row), passed to every kernel as
// an argument.
// The grid is stored order-major: for each order L and grid point i the
// kBoysTaylor values F_L..F_{L+7}(T0_i) are one aligned 64-byte row
// (table + (L kBoysGrid + i) kBoysTaylor), read with four 16-byte loads.
__device__ __forceinline__ void boys_row(const double* __restrict__ table, int L, int i, double* c) {
    const double2* r = reinterpret_cast<const double2*>(table + ((size_t)L * kBoysGrid + i) * kBoysTaylor);
#pragma unroll
    for (int k = 0; k < kBoysTaylor / 2; k++) {
        const double2 v = __ldg(r + k);
        c[2 * k] = v.x;
        c[2 * k + 1] = v.y;
    }
}

template <int L>
__device__ __forceinline__ void boys(const double* __restrict__ table, double T, double* F) {
    static_assert(L >= 0 && L <= kMaxBoysM, "Boys order out of range");
    const double eT = exp(-T);
    if (T < kBoysTMax) {
        const int i = __double2int_rn(T * kBoysInvStep);
        const double d = T - i * kBoysStep;
        double c[kBoysTaylor];
        boys_row(table, L, i, c);
        double acc = c[kBoysTaylor - 1];
#pragma unroll
        for (int k = kBoysTaylor - 1; k >= 1; k--) acc = fma(-d * (1.0 / k), acc, c[k - 1]);
        F[L] = acc;
        const double twoT = 2.0 * T;
#pragma unroll
        for (int m = L - 1; m >= 0; m--) F[m] = fma(twoT, F[m + 1], eT) * (1.0 / (2 * m + 1));
    } else {
        const double inv = 1.0 / T;
        F[0] = 0.88622692545275801365 * sqrt(inv);  // sqrt(pi)/2 / sqrt(T)
        const double half_inv = 0.5 * inv;
#pragma unroll
        for (int m = 0; m < L; m++) F[m + 1] = fma((double)(2 * m + 1), F[m], -eT) * half_inv;
    }
}

// 1/n for n = 0..2 kMaxBoysM + 1 (entry 0 unused): the run-time variant's
// recursion factors as multiplications, the same as the compile-time variant.
#define EIP_INV8(n) 1.0 / (n), 1.0 / (n + 1), 1.0 / (n + 2), 1.0 / (n + 3), 1.0 / (n + 4), 1.0 / (n + 5), \
                    1.0 / (n + 6), 1.0 / (n + 7)
static __constant__ double c_inv_n[48] = {0.0,        1.0,        0.5,        1.0 / 3,    0.25,       0.2,
                                          1.0 / 6,    1.0 / 7,    EIP_INV8(8), EIP_INV8(16), EIP_INV8(24),
                                          EIP_INV8(32), EIP_INV8(40)};
#undef EIP_INV8
static_assert(2 * kMaxBoysM + 1 < 48, "reciprocal table too short");

// Run-time order variant (generic kernels).
__device__ __forceinline__ void boys_rt(const double* __restrict__ table, int L, double T, double* F) {
    const double eT = exp(-T);
    if (T < kBoysTMax) {
        const int i = __double2int_rn(T * kBoysInvStep);
        const double d = T - i * kBoysStep;
        double c[kBoysTaylor];
        boys_row(table, L, i, c);
        double acc = c[kBoysTaylor - 1];
#pragma unroll
        for (int k = kBoysTaylor - 1; k >= 1; k--) acc = fma(-d * c_inv_n[k], acc, c[k - 1]);
        F[L] = acc;
        for (int m = L - 1; m >= 0; m--) F[m] = fma(2.0 * T, F[m + 1], eT) * c_inv_n[2 * m + 1];
    } else {
        F[0] = 0.88622692545275801365 * sqrt(1.0 / T);
        for (int m = 0; m < L; m++) F[m + 1] = fma((double)(2 * m + 1), F[m], -eT) * (0.5 / T);
    }
}

// ---------------------------------------------------------------- device tables
// Shell-pair ("bra") table of one angular class: primitive pairs grouped by
// contracted shell pair.  prim_P = (Px,Py,Pz,p); prim_PA = (PAx,PAy,PAz,coef);
// grp_AB = (ABx,ABy,ABz,0); grp_ao = (i_ao_start, j_ao_start).
struct BraTable {
    int n_group;
    const int* grp_begin;  // n_group + 1
    const int2* grp_ao;
    const double4* grp_AB;
    const double4* prim_P;
    const double4* prim_PA;
    // Optional: per primitive pair, the x, y and z tables E^{i,j}_t
    // (3 * e_size<LI,LJ>() doubles, fast (mu nu|P) kernels only).
    const double* prim_E;
};

// Work map of one (l_i, l_j | l_k) class over a batch of molecules.
// Molecule m owns shell pairs [sp_begin[m], sp_begin[m+1]) of the class's
// bra table and auxiliary shells [aux_begin[m], aux_begin[m+1]) of its ket
// table.  Its work items are (shell pair, tile of 32 auxiliary shells),
// numbered from item_begin[m]; its packed output block starts at element
// out_begin[m].  checksum (optional) receives the sum of every value written
// for molecule m.
//
// Optional shell-pair list (mixed precision: the FP32 and FP64 kernels of a
// class each take a subset of the shell pairs): when sp_list is set, molecule
// m's k-th pair is sp_list[sp_begin[m] + k] (a global index) and its output
// row is that index minus sp_first[m], the molecule's first pair.
//
// Optional auxiliary window: when aux_count is set, molecule m's auxiliary
// shells are [aux_begin[m], aux_begin[m] + aux_count[m]) (a run over a window
// of each molecule's auxiliary basis) instead of up to aux_begin[m + 1].
struct BatchMap {
    int n_mol;
    const int* item_begin;  // n_mol + 1
    const int* sp_begin;    // n_mol + 1
    const int* aux_begin;   // n_mol + 1 (n_mol with aux_count)
    const long long* out_begin;
    double* checksum;
    const int* sp_list;   // optional
    const int* sp_first;  // n_mol, with sp_list
    const int* aux_count = nullptr;  // optional, n_mol
};

// One-centre ("ket") table: auxiliary shells of one class (or point charges).
// prim_C = (Cx,Cy,Cz,exponent); prim_coef; grp_start = first aux function.
struct KetTable {
    int n_group;
    const int* grp_begin;  // n_group + 1
    const int* grp_start;
    const double4* prim_C;
    const double* prim_coef;
};

// 2 pi^(5/2)
constexpr double kTwoPi52 = 34.986836655249725693;
constexpr double kPi = 3.14159265358979323846;

}  // namespace eip
