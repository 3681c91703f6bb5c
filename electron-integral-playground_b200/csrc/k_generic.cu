// Generic kernels: any supported angular class with run-time angular momenta.
//
// They cover what the fast templated kernels do not (Cartesian output,
// (mu nu|P) classes beyond d-d|g, every (P|Q) and nuclear-attraction class) and
// are the correctness fallback for the whole C ABI range (orbital l <= 6,
// auxiliary l <= 9; reference c_library/angular.h:3-4).
//
// raw_kernel: one CTA per (bra group, ket group, ket-Cartesian chunk); it
// accumulates the raw Cartesian block
//   raw[ij][kc] = sum_prims pref * sum_{tuv} E^{ij}_{tuv} sum_s (-1)^{|s|} E^{kc}_s R_{tuv+s}
// in shared memory (stages: Boys -> R tetrahedron -> ket Hermite X[h][kc] ->
// bra contraction) and stores it to a scratch buffer
//   raw[((bra * n_ket + ket) * NIJ + ij) * NKC + kc].
// Modes: three-centre / two-centre (one-centre bra: LJ = 0 and PA = AB = 0) use
// the Coulomb prefactor 2 pi^{5/2}/(p q sqrt(p+q)) (MI/three_center.cpp:46-49,
// MI/two_center.cpp:34-37); point charges use 2 pi / p with zeta = p
// (MI/nuclear_attraction.cpp:44-45, :69).
//
// transform_kernel: raw Cartesian blocks -> spherical (real solid harmonics)
// or per-component-normalised Cartesian output, written in the packed layout
//   out[((bra * n_io * n_jo + I * n_jo + J) * n_ko + K) * n_ket + ket].
#include <algorithm>

#include "eip_common.cuh"
#include "eip_internal.h"

namespace eip {

__constant__ double c_sph_coef[sizeof(eip_sph_coef) / sizeof(double)];
__constant__ int c_sph_offset[EIP_SPH_LMAX + 2];
__constant__ double c_cart_norm[sizeof(eip_cart_norm) / sizeof(double)];
__constant__ int c_cart_norm_offset[EIP_SPH_LMAX + 2];

int upload_generic_tables() {
    cudaError_t e = cudaMemcpyToSymbol(c_sph_coef, eip_sph_coef, sizeof(eip_sph_coef));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_sph_offset, eip_sph_offset, sizeof(eip_sph_offset));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_cart_norm, eip_cart_norm, sizeof(eip_cart_norm));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_cart_norm_offset, eip_cart_norm_offset, sizeof(eip_cart_norm_offset));
    return e == cudaSuccess ? 0 : (int)e;
}

__device__ __forceinline__ void herm_decode(int idx, int& t, int& u, int& v) {
    int N = 0;
    while (nherm(N) <= idx) N++;
    int r = idx - nherm(N - 1);
    // r-th component of order N in x-major descending order
    int a = N;
    while (r > N - a) {
        r -= N - a + 1;
        a--;
    }
    t = a;
    u = N - a - r;
    v = N - t - u;
}

__device__ __forceinline__ void cart_decode(int l, int c, int& x, int& y, int& z) {
    int a = l, r = c;
    while (r > l - a) {
        r -= l - a + 1;
        a--;
    }
    x = a;
    y = l - a - r;
    z = l - x - y;
}

__device__ __forceinline__ double rt_one_centre(int k, int s) {
    if (s < 0 || s > k || ((k - s) & 1)) return 0.0;
    int h = (k - s) / 2;
    double r = 1.0;
    for (int i = 2; i <= k; i++) r *= i;
    for (int i = 2; i <= h; i++) r /= i;
    for (int i = 2; i <= s; i++) r /= i;
    for (int i = 0; i < h; i++) r *= 0.5;
    return r;
}

__device__ __forceinline__ double rt_hermite_r(int t, int m) {
    if (m < (t + 1) / 2 || m > t) return 0.0;
    double r = 1.0;
    for (int i = 2; i <= t; i++) r *= i;
    for (int i = 2; i <= 2 * m - t; i++) r /= i;
    for (int i = 2; i <= t - m; i++) r /= i;
    for (int i = 0; i < t - m; i++) r *= 0.5;
    return r;
}

constexpr int kGenThreads = 128;

struct GenericShape {
    int LI, LJ, LK, L, LIJ;
    int NI, NJ, NIJ, NKC, NR, NHB, NE, kc_chunk;
};

__host__ __device__ inline GenericShape generic_shape(int li, int lj, int lk, int kc_chunk) {
    GenericShape g;
    g.LI = li; g.LJ = lj; g.LK = lk; g.L = li + lj + lk; g.LIJ = li + lj;
    g.NI = ncart(li); g.NJ = ncart(lj); g.NIJ = g.NI * g.NJ; g.NKC = ncart(lk);
    g.NR = nherm(g.L); g.NHB = nherm(g.LIJ);
    g.NE = (li + 1) * (lj + 1) * (li + lj + 1);
    g.kc_chunk = kc_chunk;
    return g;
}

size_t generic_smem_bytes(int li, int lj, int lk, int kc_chunk) {
    GenericShape g = generic_shape(li, lj, lk, kc_chunk);
    size_t n = g.NR + (g.L + 1) + 8 + 3 * g.NE + (g.LK + 1) * (g.LK + 1) + (size_t)g.NHB * kc_chunk +
               (size_t)g.NIJ * kc_chunk;
    return n * sizeof(double);
}

// mode: 0 Coulomb (three-centre or two-centre), 1 point charges.
__global__ void __launch_bounds__(kGenThreads)
raw_kernel(const double* __restrict__ boys_table, int mode, int li, int lj, int lk, int kc_chunk, BraTable bra,
           KetTable ket, double omega, int skip_lower, double* __restrict__ raw) {
    extern __shared__ double sm[];
    const GenericShape g = generic_shape(li, lj, lk, kc_chunk);
    const int ib = blockIdx.x, ik = blockIdx.y, chunk = blockIdx.z;
    const int kc0 = chunk * kc_chunk;
    const int nkc = min(kc_chunk, g.NKC - kc0);
    if (skip_lower && bra.grp_ao[ib].x > ket.grp_start[ik]) return;

    double* sR = sm;
    double* sRm = sR + g.NR;
    double* sPar = sRm + g.L + 1;  // [0] pref
    double* sE = sPar + 8;         // 3 * NE, index (i*(LJ+1)+j)*(LIJ+1)+t
    double* sEk = sE + 3 * g.NE;   // (LK+1)^2: E^{k}_s(q)
    double* sX = sEk + (g.LK + 1) * (g.LK + 1);
    double* sJ = sX + (size_t)g.NHB * kc_chunk;
    const int tid = threadIdx.x;
    for (int e = tid; e < g.NIJ * kc_chunk; e += kGenThreads) sJ[e] = 0.0;

    const int pb = bra.grp_begin[ib], pe = bra.grp_begin[ib + 1];
    const int kb = ket.grp_begin[ik], ke = ket.grp_begin[ik + 1];
    const double4 AB = bra.grp_AB[ib];
    for (int pp = pb; pp < pe; pp++) {
        const double4 P = bra.prim_P[pp];
        const double4 PA = bra.prim_PA[pp];
        const double p = P.w;
        for (int kp = kb; kp < ke; kp++) {
            __syncthreads();
            const double4 Cq = ket.prim_C[kp];
            if (tid == 0) {
                const double X = P.x - Cq.x, Y = P.y - Cq.y, Z = P.z - Cq.z;
                double zeta, pref;
                if (mode == 0) {
                    const double q = Cq.w;
                    if (omega == 0.0) {
                        zeta = p * q / (p + q);
                        pref = PA.w * ket.prim_coef[kp] * kTwoPi52 / (p * q * sqrt(p + q));
                    } else {
                        zeta = 1.0 / (1.0 / p + 1.0 / q + 1.0 / (omega * omega));
                        pref = PA.w * ket.prim_coef[kp] * kTwoPi52 * omega /
                               (p * q * sqrt(p * q + (p + q) * omega * omega));
                    }
                } else {
                    if (omega == 0.0) {
                        zeta = p;
                        pref = PA.w * ket.prim_coef[kp] * 2.0 * kPi / p;
                    } else {
                        zeta = p * omega * omega / (p + omega * omega);
                        pref = PA.w * ket.prim_coef[kp] * 2.0 * kPi * omega / (p * sqrt(p + omega * omega));
                    }
                }
                double F[kMaxBoysM + 1];
                boys_rt(boys_table, g.L, zeta * (X * X + Y * Y + Z * Z), F);
                double f = 1.0;
                for (int m = 0; m <= g.L; m++) {
                    sRm[m] = f * F[m];
                    f *= -2.0 * zeta;
                }
                sPar[0] = pref;
                sPar[1] = X; sPar[2] = Y; sPar[3] = Z;
            } else if (tid >= 32 && tid < 35) {
                const int d = tid - 32;
                const double pa = d == 0 ? PA.x : (d == 1 ? PA.y : PA.z);
                const double ab = d == 0 ? AB.x : (d == 1 ? AB.y : AB.z);
                const double inv2p = 0.5 / p;
                const int N = g.LIJ;
                double W[13][7][13];  // i <= 12, j <= 6, t <= 12
                for (int i = 0; i <= N; i++)
                    for (int j = 0; j <= g.LJ; j++)
                        for (int t = 0; t <= N; t++) W[i][j][t] = 0.0;
                W[0][0][0] = 1.0;
                for (int i = 0; i < N; i++)
                    for (int t = 0; t <= i + 1; t++) {
                        double v = 0.0;
                        if (t >= 1) v = inv2p * W[i][0][t - 1];
                        if (t <= i) v = fma(pa, W[i][0][t], v);
                        if (t + 1 <= i) v = fma((double)(t + 1), W[i][0][t + 1], v);
                        W[i + 1][0][t] = v;
                    }
                for (int j = 0; j < g.LJ; j++)
                    for (int i = 0; i + j + 1 <= N; i++)
                        for (int t = 0; t <= i + j + 1; t++) W[i][j + 1][t] = fma(ab, W[i][j][t], W[i + 1][j][t]);
                double* out = sE + d * g.NE;
                for (int i = 0; i <= g.LI; i++)
                    for (int j = 0; j <= g.LJ; j++)
                        for (int t = 0; t <= N; t++) out[(i * (g.LJ + 1) + j) * (N + 1) + t] = W[i][j][t];
            } else if (tid == 64) {
                const double inv2q = mode == 0 ? 0.5 / Cq.w : 0.0;
                for (int k = 0; k <= g.LK; k++)
                    for (int s = 0; s <= g.LK; s++) {
                        double c = rt_one_centre(k, s);
                        for (int i = 0; i < (k + s) / 2; i++) c *= inv2q;
                        sEk[k * (g.LK + 1) + s] = c;
                    }
            }
            __syncthreads();
            {
                const double X = sPar[1], Y = sPar[2], Z = sPar[3];
                for (int idx = tid; idx < g.NR; idx += kGenThreads) {
                    int t, u, v;
                    herm_decode(idx, t, u, v);
                    double r = 0.0;
                    for (int mx = (t + 1) / 2; mx <= t; mx++) {
                        double ry = 0.0;
                        for (int my = (u + 1) / 2; my <= u; my++) {
                            double rz = 0.0;
                            for (int mz = (v + 1) / 2; mz <= v; mz++)
                                rz = fma(rt_hermite_r(v, mz) * pow(Z, (double)(2 * mz - v)), sRm[mx + my + mz], rz);
                            ry = fma(rt_hermite_r(u, my) * pow(Y, (double)(2 * my - u)), rz, ry);
                        }
                        r = fma(rt_hermite_r(t, mx) * pow(X, (double)(2 * mx - t)), ry, r);
                    }
                    sR[idx] = r;
                }
            }
            __syncthreads();
            for (int e = tid; e < g.NHB * nkc; e += kGenThreads) {
                const int h = e / nkc, c = e - h * nkc;
                int t, u, v, kx, ky, kz;
                herm_decode(h, t, u, v);
                cart_decode(g.LK, kc0 + c, kx, ky, kz);
                double x = 0.0;
                for (int sx = kx & 1; sx <= kx; sx += 2)
                    for (int sy = ky & 1; sy <= ky; sy += 2)
                        for (int sz = kz & 1; sz <= kz; sz += 2) {
                            const double ek = sEk[kx * (g.LK + 1) + sx] * sEk[ky * (g.LK + 1) + sy] *
                                              sEk[kz * (g.LK + 1) + sz];
                            const double r = sR[herm_index(t + sx, u + sy, v + sz)];
                            x = ((sx + sy + sz) & 1) ? fma(-ek, r, x) : fma(ek, r, x);
                        }
                sX[h * kc_chunk + c] = x;
            }
            __syncthreads();
            const double pref = sPar[0];
            const int N1 = g.LIJ + 1;
            for (int e = tid; e < g.NIJ * nkc; e += kGenThreads) {
                const int ij = e / nkc, c = e - ij * nkc;
                const int ci = ij / g.NJ, cj = ij - ci * g.NJ;
                int ix, iy, iz, jx, jy, jz;
                cart_decode(g.LI, ci, ix, iy, iz);
                cart_decode(g.LJ, cj, jx, jy, jz);
                const double* ex = sE + (ix * (g.LJ + 1) + jx) * N1;
                const double* ey = sE + g.NE + (iy * (g.LJ + 1) + jy) * N1;
                const double* ez = sE + 2 * g.NE + (iz * (g.LJ + 1) + jz) * N1;
                double s = 0.0;
                for (int t = 0; t <= ix + jx; t++) {
                    double su = 0.0;
                    for (int u = 0; u <= iy + jy; u++) {
                        double sv = 0.0;
                        for (int v = 0; v <= iz + jz; v++) sv = fma(ez[v], sX[herm_index(t, u, v) * kc_chunk + c], sv);
                        su = fma(ey[u], sv, su);
                    }
                    s = fma(ex[t], su, s);
                }
                sJ[ij * kc_chunk + c] = fma(pref, s, sJ[ij * kc_chunk + c]);
            }
        }
    }
    __syncthreads();
    const size_t base = ((size_t)ib * ket.n_group + ik) * g.NIJ;
    for (int e = tid; e < g.NIJ * nkc; e += kGenThreads) {
        const int ij = e / nkc, c = e - ij * nkc;
        raw[(base + ij) * g.NKC + kc0 + c] = sJ[ij * kc_chunk + c];
    }
}

// Overlap: one thread per (shell pair, ci, cj) raw Cartesian element;
// S = c (pi/p)^{3/2} E^{ix,jx}_0 E^{iy,jy}_0 E^{iz,jz}_0 (MI/overlap.cpp:10-16),
// PA = -b/p AB as in MI/overlap.cpp:21-28.
__global__ void overlap_raw_kernel(int li, int lj, BraTable bra, const double* __restrict__ prim_b,
                                   double* __restrict__ raw) {
    const int NI = ncart(li), NJ = ncart(lj), NIJ = NI * NJ;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)bra.n_group * NIJ) return;
    const int ib = (int)(e / NIJ), ij = (int)(e - (long long)ib * NIJ);
    const int ci = ij / NJ, cj = ij - ci * NJ;
    int ax[3], bx[3];
    cart_decode(li, ci, ax[0], ax[1], ax[2]);
    cart_decode(lj, cj, bx[0], bx[1], bx[2]);
    const double4 AB = bra.grp_AB[ib];
    const double abv[3] = {AB.x, AB.y, AB.z};
    double acc = 0.0;
    for (int pp = bra.grp_begin[ib]; pp < bra.grp_begin[ib + 1]; pp++) {
        const double p = bra.prim_P[pp].w;
        const double b = prim_b[pp];
        const double inv2p = 0.5 / p;
        double prod = bra.prim_PA[pp].w * pow(kPi / p, 1.5);
        for (int d = 0; d < 3; d++) {
            const double pa = -b / p * abv[d];
            const int i = ax[d], j = bx[d], N = i + j;
            double V[13][13];
            for (int a = 0; a <= N; a++)
                for (int t = 0; t <= N; t++) V[a][t] = 0.0;
            V[0][0] = 1.0;
            for (int a = 0; a < N; a++)
                for (int t = 0; t <= a + 1; t++) {
                    double v = 0.0;
                    if (t >= 1) v = inv2p * V[a][t - 1];
                    if (t <= a) v = fma(pa, V[a][t], v);
                    if (t + 1 <= a) v = fma((double)(t + 1), V[a][t + 1], v);
                    V[a + 1][t] = v;
                }
            // E^{i,j}_0 = sum_m binom(j, m) AB^{j-m} E^{i+m,0}_0
            double ej = 0.0, abp = 1.0, binom = 1.0;
            for (int m = j; m >= 0; m--) {
                ej = fma(binom * abp, V[i + m][0], ej);
                abp *= abv[d];
                binom = binom * m / (j - m + 1);
            }
            prod *= ej;
        }
        acc += prod;
    }
    raw[e] = acc;
}

__device__ __forceinline__ double rt_out_coef(bool spherical, int l, int o, int c) {
    if (spherical) return c_sph_coef[c_sph_offset[l] + o * ncart(l) + c];
    return o == c ? c_cart_norm[c_cart_norm_offset[l] + c] : 0.0;
}

// raw[bra][ket][ci*NJ+cj][kc] -> out[((bra*n_io*n_jo + I*n_jo + J)*n_ko + K)*n_ket + ket]
__global__ void transform_kernel(int li, int lj, int lk, bool spherical, int n_bra, int n_ket,
                                 const double* __restrict__ raw, double* __restrict__ out) {
    const int NI = ncart(li), NJ = ncart(lj), NK = ncart(lk);
    const int n_io = spherical ? nsph(li) : NI, n_jo = spherical ? nsph(lj) : NJ, n_ko = spherical ? nsph(lk) : NK;
    const long long total = (long long)n_bra * n_io * n_jo * n_ko * n_ket;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long r = e;
        const int ket = (int)(r % n_ket); r /= n_ket;
        const int K = (int)(r % n_ko); r /= n_ko;
        const int J = (int)(r % n_jo); r /= n_jo;
        const int I = (int)(r % n_io); r /= n_io;
        const int bra = (int)r;
        const double* blk = raw + ((size_t)bra * n_ket + ket) * NI * NJ * NK;
        double v = 0.0;
        for (int ci = 0; ci < NI; ci++) {
            const double wi = rt_out_coef(spherical, li, I, ci);
            if (wi == 0.0) continue;
            for (int cj = 0; cj < NJ; cj++) {
                const double wj = rt_out_coef(spherical, lj, J, cj);
                if (wj == 0.0) continue;
                double vk = 0.0;
                for (int ck = 0; ck < NK; ck++) {
                    const double wk = rt_out_coef(spherical, lk, K, ck);
                    if (wk != 0.0) vk = fma(wk, blk[(ci * NJ + cj) * NK + ck], vk);
                }
                v = fma(wi * wj, vk, v);
            }
        }
        out[e] = v;
    }
}

int generic_kc_chunk(int li, int lj, int lk) {
    const int NKC = ncart(lk), NIJ = ncart(li) * ncart(lj), NHB = nherm(li + lj);
    int chunk = NKC;
    while (chunk > 1 && (size_t)(NIJ + NHB) * chunk > 12000) chunk = (chunk + 1) / 2;
    return chunk;
}

// Largest dynamic shared memory raw_kernel takes over every class the C ABI
// accepts (orbital l <= 6, auxiliary l <= 9; the two-centre bra up to l = 9).
static size_t generic_max_smem() {
    size_t m = 0;
    for (int li = 0; li <= kMaxAuxL; li++)
        for (int lj = 0; lj <= kMaxOrbitalL; lj++)
            for (int lk = 0; lk <= kMaxAuxL; lk++)
                if (li + lj + lk <= kMaxBoysM) m = std::max(m, generic_smem_bytes(li, lj, lk, generic_kc_chunk(li, lj, lk)));
    return m;
}

int launch_generic_raw(int mode, int li, int lj, int lk, const BraTable& bra, const KetTable& ket, double omega,
                       int skip_lower, double* raw, cudaStream_t s) {
    if (bra.n_group == 0 || ket.n_group == 0) return 0;
    const int chunk = generic_kc_chunk(li, lj, lk);
    const int n_chunks = (ncart(lk) + chunk - 1) / chunk;
    const size_t smem = generic_smem_bytes(li, lj, lk, chunk);
    // the shared-memory limit is raised once per device, to the largest class's
    // need (persistent_grid caches per device and serialises the set-up)
    static std::atomic<int> configured[kMaxDevices];
    if (persistent_grid(reinterpret_cast<const void*>(raw_kernel), kGenThreads, generic_max_smem(), configured) <= 0)
        return 2;
    const double* table = boys_table_device();
    if (!table) return 2;
    if (ket.n_group > 65535) return 3;
    dim3 grid(bra.n_group, ket.n_group, n_chunks);
    raw_kernel<<<grid, kGenThreads, smem, s>>>(table, mode, li, lj, lk, chunk, bra, ket, omega, skip_lower, raw);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int launch_overlap_raw(int li, int lj, const BraTable& bra, const double* prim_b, double* raw, cudaStream_t s) {
    const long long total = (long long)bra.n_group * ncart(li) * ncart(lj);
    if (total == 0) return 0;
    overlap_raw_kernel<<<(unsigned)((total + 127) / 128), 128, 0, s>>>(li, lj, bra, prim_b, raw);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int launch_transform(int li, int lj, int lk, bool spherical, int n_bra, int n_ket, const double* raw, double* out,
                     cudaStream_t s) {
    const long long total = (long long)n_bra * n_ket * (spherical ? nsph(li) * nsph(lj) * nsph(lk)
                                                                  : ncart(li) * ncart(lj) * ncart(lk));
    if (total == 0) return 0;
    long long blocks = (total + 255) / 256;
    if (blocks > 148 * 64) blocks = 148 * 64;
    transform_kernel<<<(unsigned)blocks, 256, 0, s>>>(li, lj, lk, spherical, n_bra, n_ket, raw, out);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace eip
