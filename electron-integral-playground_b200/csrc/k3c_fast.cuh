// Fast (mu nu|P) kernels for the common low-angular-momentum classes.
//
// Computes, for every contracted shell pair (mu nu) of one (l_i, l_j) class and
// every auxiliary shell P of class l_k, the spherical block
//   (mu nu|P) = sum_{prim pairs} sum_{aux prims} c_ab c_P 2 pi^{5/2} / (p q sqrt(p+q))
//               sum_{tuv} E^{ij}_{tuv} sum_{s} (-1)^{|s|} E^{k}_{s}(q) R_{t+s_x,u+s_y,v+s_z}
// (reference: MI/three_center.cpp:10-26 for the formula, :27-173 for one
// primitive triplet; erf-attenuated variant for omega > 0, :46-49).
//
// Mapping (this library's design, not the reference's): one CTA handles one
// shell pair and 32 auxiliary shells, lane = auxiliary shell, so the final
// stores of each warp are 32 consecutive doubles.  The KS warps of the CTA
// split (a) the entries of the Hermite tetrahedron R_{tuv} (closed form from
// R^{(m)}_000, written to shared memory) and (b) the spherical ket
// components; the ket Cartesian->spherical transform and the one-centre
// Hermite coefficients are folded into compile-time constants.  Primitive
// pairs are reduced in registers: each contracted block is written once, with
// no atomics.  Output layout ("packed"):
//   out[((pair * nsph_i * nsph_j + I * nsph_j + J) * nsph_k + K) * n_aux_shell + P]
#pragma once

#include "eip_common.cuh"
#include "eip_internal.h"

namespace eip {

constexpr int kAccMax = 48;  // accumulators (doubles) per lane

template <int LI, int LJ, int LK>
struct Fast3c {
    static constexpr int L = LI + LJ + LK;
    static constexpr int LIJ = LI + LJ;
    static constexpr int NI = ncart(LI), NJ = ncart(LJ), NIJ = NI * NJ;
    static constexpr int NKO = nsph(LK);
    static constexpr int KPW_MAX = (kAccMax / NIJ) < 1 ? 1 : (kAccMax / NIJ);
    static constexpr int KS = (NKO + KPW_MAX - 1) / KPW_MAX;  // warps per CTA
    static constexpr int KPW = (NKO + KS - 1) / KS;           // ket components per warp
    static constexpr int NR = nherm(L);
    static constexpr int RPW = (NR + KS - 1) / KS;            // R entries per warp
    static constexpr int NHB = nherm(LIJ);
    static constexpr int NE = e_size<LI, LJ>();
    static constexpr int THREADS = 32 * KS;
};

// Two-centre E^{i,j}_t along one axis for i <= LI, j <= LJ:
// vertical recursion E^{i+1,0}_t = E^{i,0}_{t-1}/(2p) + PA E^{i,0}_t + (t+1) E^{i,0}_{t+1},
// then transfer E^{i,j+1}_t = E^{i+1,j}_t + AB E^{i,j}_t.
template <int LI, int LJ>
__device__ __forceinline__ void bra_e_table(double PA, double AB, double inv2p, double* out) {
    constexpr int N = LI + LJ;
    double W[N + 1][LJ + 1][N + 1];
#pragma unroll
    for (int i = 0; i <= N; i++)
#pragma unroll
        for (int j = 0; j <= LJ; j++)
#pragma unroll
            for (int t = 0; t <= N; t++) W[i][j][t] = 0.0;
    W[0][0][0] = 1.0;
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int t = 0; t <= i + 1; t++) {
            double v = 0.0;
            if (t >= 1) v = inv2p * W[i][0][t - 1];
            if (t <= i) v = fma(PA, W[i][0][t], v);
            if (t + 1 <= i) v = fma((double)(t + 1), W[i][0][t + 1], v);
            W[i + 1][0][t] = v;
        }
#pragma unroll
    for (int j = 0; j < LJ; j++)
#pragma unroll
        for (int i = 0; i + j + 1 <= N; i++)
#pragma unroll
            for (int t = 0; t <= i + j + 1; t++) W[i][j + 1][t] = fma(AB, W[i][j][t], W[i + 1][j][t]);
#pragma unroll
    for (int i = 0; i <= LI; i++)
#pragma unroll
        for (int j = 0; j <= LJ; j++)
#pragma unroll
            for (int t = 0; t <= i + j; t++) out[e_offset<LJ>(i, j) + t] = W[i][j][t];
}

template <int LI, int LJ, int LK>
__global__ void __launch_bounds__(Fast3c<LI, LJ, LK>::THREADS)
k3c_fast(const double* __restrict__ boys_table, BraTable bra, KetTable ket, int n_tiles, double omega,
         double* __restrict__ out) {
    using C = Fast3c<LI, LJ, LK>;
    constexpr int L = C::L;
    __shared__ double sE[3 * C::NE];
    __shared__ double sR[C::NR * 32];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int sp = blockIdx.x / n_tiles;
    const int tile = blockIdx.x - sp * n_tiles;
    const int a = tile * 32 + lane;
    const bool valid = a < ket.n_group;
    int kb = 0, nk = 0;
    if (valid) {
        kb = ket.grp_begin[a];
        nk = ket.grp_begin[a + 1] - kb;
    }
    const int nk_max = __reduce_max_sync(0xffffffffu, nk);
    const int pb = bra.grp_begin[sp], pe = bra.grp_begin[sp + 1];
    const double4 AB = bra.grp_AB[sp];

    double acc[C::NIJ][C::KPW];
#pragma unroll
    for (int i = 0; i < C::NIJ; i++)
#pragma unroll
        for (int c = 0; c < C::KPW; c++) acc[i][c] = 0.0;

    for (int pp = pb; pp < pe; pp++) {
        const double4 P = bra.prim_P[pp];
        const double4 PA = bra.prim_PA[pp];
        const double p = P.w;
        if (warp == 0 && lane < 3) {
            const double pa = lane == 0 ? PA.x : (lane == 1 ? PA.y : PA.z);
            const double ab = lane == 0 ? AB.x : (lane == 1 ? AB.y : AB.z);
            bra_e_table<LI, LJ>(pa, ab, 0.5 / p, sE + lane * C::NE);
        }
        for (int kk = 0; kk < nk_max; kk++) {
            const bool live = kk < nk;
            const double4 Cq = live ? ket.prim_C[kb + kk] : make_double4(P.x, P.y, P.z, 1.0);
            const double cc = live ? ket.prim_coef[kb + kk] : 0.0;
            const double q = Cq.w;
            const double X = P.x - Cq.x, Y = P.y - Cq.y, Z = P.z - Cq.z;
            double zeta, pref;
            if (omega == 0.0) {
                zeta = p * q / (p + q);
                pref = PA.w * cc * kTwoPi52 / (p * q * sqrt(p + q));
            } else {
                zeta = 1.0 / (1.0 / p + 1.0 / q + 1.0 / (omega * omega));
                pref = PA.w * cc * kTwoPi52 * omega / (p * q * sqrt(p * q + (p + q) * omega * omega));
            }
            if (LK & 1) pref = -pref;  // (-1)^{|s|} with |s| = LK mod 2

            // R^{(m)}_000 = (-2 zeta)^m F_m(zeta |PQ|^2), then this warp's share of
            // the tetrahedron by the closed form (per-entry independent).
            double Rm[L + 1];
            boys<L>(boys_table, zeta * (X * X + Y * Y + Z * Z), Rm);
            {
                double f = -2.0 * zeta, g = f;
#pragma unroll
                for (int m = 1; m <= L; m++) {
                    Rm[m] *= g;
                    g *= f;
                }
            }
            double px[L + 1], py[L + 1], pz[L + 1];
            px[0] = py[0] = pz[0] = 1.0;
#pragma unroll
            for (int m = 1; m <= L; m++) {
                px[m] = px[m - 1] * X;
                py[m] = py[m - 1] * Y;
                pz[m] = pz[m - 1] * Z;
            }
            static_for<0, C::KS>([&](auto g) {
                constexpr int G = decltype(g)::value;
                constexpr int lo = G * C::RPW;
                constexpr int hi = (G + 1) * C::RPW < C::NR ? (G + 1) * C::RPW : C::NR;
                if (warp == G) {
                    static_for<lo, hi>([&](auto e) {
                        constexpr int idx = decltype(e)::value;
                        constexpr int t = herm_t(idx), u = herm_u(idx), v = herm_v(idx);
                        double r = 0.0;
                        static_for<(t + 1) / 2, t + 1>([&](auto mx_) {
                            constexpr int mx = decltype(mx_)::value;
                            double ry = 0.0;
                            static_for<(u + 1) / 2, u + 1>([&](auto my_) {
                                constexpr int my = decltype(my_)::value;
                                double rz = 0.0;
                                static_for<(v + 1) / 2, v + 1>([&](auto mz_) {
                                    constexpr int mz = decltype(mz_)::value;
                                    constexpr double h = hermite_r_coef(v, mz);
                                    rz = fma(h * pz[2 * mz - v], Rm[mx + my + mz], rz);
                                });
                                constexpr double h = hermite_r_coef(u, my);
                                ry = fma(h * py[2 * my - u], rz, ry);
                            });
                            constexpr double h = hermite_r_coef(t, mx);
                            r = fma(h * px[2 * mx - t], ry, r);
                        });
                        sR[idx * 32 + lane] = r;
                    });
                }
            });
            // (1/2q)^{LK - j} weights of |s| = LK - 2j
            double w[LK / 2 + 1];
            {
                const double inv2q = 0.5 / q;
                double base = 1.0;
#pragma unroll
                for (int j = 0; j < LK - LK / 2; j++) base *= inv2q;
                // base = (1/2q)^{ceil(LK/2)} = weight of j = LK/2
#pragma unroll
                for (int j = LK / 2; j >= 0; j--) {
                    w[j] = base;
                    base *= inv2q;
                }
            }
            __syncthreads();

            static_for<0, C::KS>([&](auto g) {
                constexpr int G = decltype(g)::value;
                if (warp == G) {
                    static_for<0, C::KPW>([&](auto c_) {
                        constexpr int c = decltype(c_)::value;
                        constexpr int ko = G * C::KPW + c;
                        if constexpr (ko < C::NKO) {
                            double Xh[C::NHB];
                            static_for<0, C::NHB>([&](auto h_) {
                                constexpr int h = decltype(h_)::value;
                                constexpr int t = herm_t(h), u = herm_u(h), v = herm_v(h);
                                double xs = 0.0;
                                static_for<0, LK / 2 + 1>([&](auto j_) {
                                    constexpr int j = decltype(j_)::value;
                                    constexpr int S = LK - 2 * j;
                                    double part = 0.0;
                                    static_for<0, ncart(S)>([&](auto sc_) {
                                        constexpr int sc = decltype(sc_)::value;
                                        constexpr int sx = cart_x(S, sc), sy = cart_y(S, sc), sz = cart_z(S, sc);
                                        constexpr double kc = ket_sph_coef(LK, ko, sx, sy, sz);
                                        if constexpr (kc != 0.0)
                                            part = fma(kc, sR[herm_index(t + sx, u + sy, v + sz) * 32 + lane], part);
                                    });
                                    xs = fma(w[j], part, xs);
                                });
                                Xh[h] = xs;
                            });
                            static_for<0, C::NI>([&](auto ci_) {
                                constexpr int ci = decltype(ci_)::value;
                                constexpr int ix = cart_x(LI, ci), iy = cart_y(LI, ci), iz = cart_z(LI, ci);
                                static_for<0, C::NJ>([&](auto cj_) {
                                    constexpr int cj = decltype(cj_)::value;
                                    constexpr int jx = cart_x(LJ, cj), jy = cart_y(LJ, cj), jz = cart_z(LJ, cj);
                                    double s = 0.0;
                                    static_for<0, ix + jx + 1>([&](auto t_) {
                                        constexpr int t = decltype(t_)::value;
                                        double su = 0.0;
                                        static_for<0, iy + jy + 1>([&](auto u_) {
                                            constexpr int u = decltype(u_)::value;
                                            double sv = 0.0;
                                            static_for<0, iz + jz + 1>([&](auto v_) {
                                                constexpr int v = decltype(v_)::value;
                                                sv = fma(sE[2 * C::NE + e_offset<LJ>(iz, jz) + v], Xh[herm_index(t, u, v)], sv);
                                            });
                                            su = fma(sE[C::NE + e_offset<LJ>(iy, jy) + u], sv, su);
                                        });
                                        s = fma(sE[e_offset<LJ>(ix, jx) + t], su, s);
                                    });
                                    acc[ci * C::NJ + cj][c] = fma(pref, s, acc[ci * C::NJ + cj][c]);
                                });
                            });
                        }
                    });
                }
            });
            __syncthreads();
        }
    }

    if (!valid) return;
    const size_t n_ket = (size_t)ket.n_group;
    static_for<0, C::KS>([&](auto g) {
        constexpr int G = decltype(g)::value;
        if (warp == G) {
            static_for<0, C::KPW>([&](auto c_) {
                constexpr int c = decltype(c_)::value;
                constexpr int ko = G * C::KPW + c;
                if constexpr (ko < C::NKO) {
                    static_for<0, nsph(LI)>([&](auto I_) {
                        constexpr int I = decltype(I_)::value;
                        static_for<0, nsph(LJ)>([&](auto J_) {
                            constexpr int J = decltype(J_)::value;
                            double v = 0.0;
                            static_for<0, C::NI>([&](auto ci_) {
                                constexpr int ci = decltype(ci_)::value;
                                constexpr double wi = sph_coef(LI, I, ci);
                                if constexpr (wi != 0.0) {
                                    double vj = 0.0;
                                    static_for<0, C::NJ>([&](auto cj_) {
                                        constexpr int cj = decltype(cj_)::value;
                                        constexpr double wj = sph_coef(LJ, J, cj);
                                        if constexpr (wj != 0.0) vj = fma(wj, acc[ci * C::NJ + cj][c], vj);
                                    });
                                    v = fma(wi, vj, v);
                                }
                            });
                            const size_t row = ((size_t)sp * nsph(LI) * nsph(LJ) + I * nsph(LJ) + J) * C::NKO + ko;
                            out[row * n_ket + a] = v;
                        });
                    });
                }
            });
        }
    });
}

template <int LI, int LJ, int LK>
static int launch_one(const double* boys_table, const BraTable& bra, const KetTable& ket, double omega, double* out,
                      cudaStream_t s) {
    using C = Fast3c<LI, LJ, LK>;
    if (bra.n_group == 0 || ket.n_group == 0) return 0;
    const int n_tiles = (ket.n_group + 31) / 32;
    const long long blocks = (long long)bra.n_group * n_tiles;
    if (blocks > 0x7fffffffLL) return 3;
    k3c_fast<LI, LJ, LK><<<(unsigned)blocks, C::THREADS, 0, s>>>(boys_table, bra, ket, n_tiles, omega, out);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace eip
