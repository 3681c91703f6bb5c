// Fast (mu nu|P) kernels for the common low-angular-momentum classes.
//
// Computes, for every contracted shell pair (mu nu) of one (l_i, l_j) class and
// every auxiliary shell P of class l_k, the spherical block
//   (mu nu|P) = sum_{prim pairs} sum_{aux prims} c_ab c_P 2 pi^{5/2} / (p q sqrt(p+q))
//               sum_{tuv} E^{ij}_{tuv} sum_{s} (-1)^{|s|} E^{k}_{s}(q) R_{t+s_x,u+s_y,v+s_z}
// (reference: MI/three_center.cpp:10-26 for the formula, :27-173 for one
// primitive triplet; erf-attenuated variant for omega > 0, :46-49).
//
// Mapping (this library's design, not the reference's):
//   * persistent CTAs take work items (shell pair, 32 auxiliary shells) of a
//     multi-molecule work list from an atomic counter;
//   * lane = auxiliary shell, so the stores of a warp are 32 consecutive doubles;
//   * the KS warps of a CTA split (a) the entries of the Hermite tetrahedron
//     R_{tuv} (closed form from R^{(m)}_000, shared through shared memory) and
//     (b) the spherical ket components (KPW per warp);
//   * the ket Cartesian->spherical transform and one-centre Hermite
//     coefficients come from a per-l_k constant-memory table (KetCoefTable),
//     so all warps run the same ket/bra code (instruction-cache friendly);
//     zero coefficients are skipped by a warp-uniform branch;
//   * E tables of each primitive pair are precomputed once into the
//     device-resident pair table (e_table_kernel) and staged per pair into
//     shared memory;
//   * FP64 kernels of pair classes with l_i > 0, l_j >= 2 accumulate the (0, b)
//     functions of the pair (l_j <= |b| <= l_i + l_j, Hermite coefficients
//     E^{0 b}_t around P of a Gaussian on centre B) and move l_i onto centre A
//     once per contracted block, in the epilogue, by the transfer
//     (a+1_d, b) = (a, b+1_d) - AB_d (a, b); AB is the same for every
//     primitive pair of a shell pair, so the transfer commutes with the
//     contraction over primitives and the per-unit bra work drops (p-d: 77
//     instead of 108 E-term products per ket component, d-d: 203 instead of
//     276).  The FP32 kernels of the mixed-precision path keep the E^{ij}_t
//     tables (transferred per primitive pair in FP64), so that no FP32
//     cancellation in the transfer enters their error budget;
//   * spherical kets read only the top Hermite level |s| = l_k of the
//     tetrahedron: a real solid harmonic is a harmonic polynomial, so the
//     Hermite expansion of its Gaussian has no lower terms (checked at compile
//     time on the coefficient tables), and tetrahedron entries of order < l_k
//     are neither computed nor stored;
//   * one-warp CTAs (most low-l classes) keep the unit's Boys values in
//     registers and load the next unit's data while evaluating the current one;
//   * primitive pairs are reduced in registers: each contracted block is
//     written once, with no atomics.
// Packed output of molecule m (element offset out_begin[m]):
//   out[((pair * nsph_i * nsph_j + I * nsph_j + J) * nsph_k + K) * n_aux_shell_m + P]
#pragma once

#include "eip_common.cuh"
#include "eip_internal.h"

namespace eip {

// Tuning variants (chosen per class by the autotuner, see autotune.py):
//   ACC   accumulators (doubles) per lane -> how many warps split the ket
//   WARPS resident warps per SM asked of the register allocator (register cap
//         65536 / (32 * WARPS)); more warps hide latency, fewer avoid spills.
//   XMAX  one-warp CTAs: the ket contraction X of at most this many values per
//         lane at a time (more components go in chunks: fewer live registers,
//         the tetrahedron read once per chunk)
//   v0 48/12 with X chunks of 24, v1 48/16 with X chunks of 24, v2 24/16, v3 96/8,
//   v4 24/24, v5 96/12 with X chunks of 24, v6 96/8 with X chunks of 24
constexpr int kVariants = 7;
__host__ __device__ constexpr int variant_acc(int v) {
    return v == 2 || v == 4 ? 24 : (v == 3 || v == 5 || v == 6 ? 96 : 48);
}
__host__ __device__ constexpr int variant_warps(int v) {
    return v == 3 || v == 6 ? 8 : (v == 0 || v == 5 ? 12 : (v == 4 ? 24 : 16));
}
__host__ __device__ constexpr int variant_xmax(int v) { return v == 2 || v == 3 || v == 4 ? 48 : 24; }

// E table record of one primitive pair (e_table_kernel): for l_i > 0, l_j >= 2 first
// E^{0 b}_t, b <= l_i + l_j, for x, y, z (the transfer-after-contraction
// kernels), then E^{i j}_t for x, y, z (the direct kernels).
template <int LI, int LJ>
__host__ __device__ constexpr int e_hrr_size() { return LI > 0 && LJ >= 2 ? (LI + LJ + 1) * (LI + LJ + 2) / 2 : 0; }
template <int LI, int LJ>
__host__ __device__ constexpr int e_record() { return 3 * (e_hrr_size<LI, LJ>() + e_size<LI, LJ>()); }

// FP64 kernels of the pair classes with l_i > 0 and l_j >= 2 transfer after
// the contraction (for p-p the saving, 27 against 33 E-term products, does not
// pay for the longer epilogue).
template <int LI, int LJ, typename T>
constexpr bool use_hrr() { return LI > 0 && LJ >= 2 && std::is_same<T, double>::value; }

// Tetrahedra of at most this many stored entries stay in registers in
// one-warp CTAs.
constexpr int kRRegMax = 20;

template <int LI, int LJ, int LK, int V = 0, bool HRR = false>
struct Fast3c {
    static constexpr int L = LI + LJ + LK;
    static constexpr int LIJ = LI + LJ;
    static constexpr int NI = ncart(LI), NJ = ncart(LJ), NIJ = NI * NJ;
    static constexpr int NIJS = nsph(LI) * nsph(LJ);
    static constexpr int NKO = nsph(LK);
    // bra functions accumulated per ket component: (0, b) functions with
    // l_j <= |b| <= l_i + l_j (transfer after contraction) or the (i, j) pairs
    static constexpr int NB = HRR ? nherm(LIJ) - nherm(LJ - 1) : NIJ;
    static constexpr int KPW_MAX = (variant_acc(V) / NB) < 1 ? 1 : (variant_acc(V) / NB);
    static constexpr int KS = (NKO + KPW_MAX - 1) / KPW_MAX;  // warps per CTA
    static constexpr int KPW = (NKO + KS - 1) / KS;           // ket components per warp
    static constexpr int NR = nherm(L);
    static constexpr int R0 = nherm(LK - 1);                  // first tetrahedron entry read by the ket
    static constexpr int NRN = NR - R0;                       // entries computed and stored
    static constexpr int RPW = (NRN + KS - 1) / KS;           // R entries per warp
    static constexpr int NHB = nherm(LIJ);
    // E entries per axis read per unit: E^{0 b}_t (transfer) or E^{i j}_t
    static constexpr int NE = HRR ? e_hrr_size<LI, LJ>() : e_size<LI, LJ>();
    // offset of those entries in a primitive pair's E record
    static constexpr int E_OFF = HRR ? 0 : 3 * e_hrr_size<LI, LJ>();
    static constexpr int THREADS = 32 * KS;
    // resident CTAs per SM asked of the register allocator
    static constexpr int MIN_CTAS = (variant_warps(V) / KS) < 1 ? 1 : (variant_warps(V) / KS);
    // units (primitive pair x auxiliary primitive) per block, doubles per unit and lane
    static constexpr int UB = KS;
    static constexpr int NU = L + 6;
    template <typename T>
    static constexpr size_t smem_bytes() {
        return (KS == 1 ? 0 : sizeof(double) * UB * NU * 32) + sizeof(T) * (NRN * 32 + UB * 3 * NE);
    }
};

// R_tuv by the closed form from R^{(m)}_000 (Rt) and the powers of PQ (px,
// py, pz): R_tuv = sum_{mx,my,mz} h(t,mx) h(u,my) h(v,mz) X^{2mx-t} Y^{2my-u}
// Z^{2mz-v} R^{(mx+my+mz)}_000.
template <int t, int u, int v, typename T>
__device__ __forceinline__ T r_closed(const T* Rt, const T* px, const T* py, const T* pz) {
    T r = T(0);
    static_for<(t + 1) / 2, t + 1>([&](auto mx_) {
        constexpr int mx = decltype(mx_)::value;
        T ry = T(0);
        static_for<(u + 1) / 2, u + 1>([&](auto my_) {
            constexpr int my = decltype(my_)::value;
            T rz = T(0);
            static_for<(v + 1) / 2, v + 1>([&](auto mz_) {
                constexpr int mz = decltype(mz_)::value;
                constexpr T h = (T)hermite_r_coef(v, mz);
                rz = fma(h * pz[2 * mz - v], Rt[mx + my + mz], rz);
            });
            constexpr T h = (T)hermite_r_coef(u, my);
            ry = fma(h * py[2 * my - u], rz, ry);
        });
        constexpr T h = (T)hermite_r_coef(t, mx);
        r = fma(h * px[2 * mx - t], ry, r);
    });
    return r;
}

// Ket coefficient table of one l_k: for spherical component ko and Hermite
// index s (|s| = LK - 2j, listed level by level in Cartesian order), the
// combined one-centre Hermite and Cartesian->spherical coefficient; the
// (1/2q)^{LK-j} weight is applied at run time.  Held in constant memory so that
// every warp runs the same ket code whatever components it owns (code
// specialised per component overflowed the instruction cache).
__host__ __device__ constexpr int ket_n_s(int LK) {
    int n = 0;
    for (int j = 0; j <= LK / 2; j++) n += ncart(LK - 2 * j);
    return n;
}
template <int LK>
struct KetCoefTable {
    double v[nsph(LK)][ket_n_s(LK)];
};
template <int LK>
constexpr KetCoefTable<LK> make_ket_table() {
    KetCoefTable<LK> t{};
    for (int ko = 0; ko < nsph(LK); ko++) {
        int idx = 0;
        for (int j = 0; j <= LK / 2; j++) {
            const int S = LK - 2 * j;
            for (int sc = 0; sc < ncart(S); sc++)
                t.v[ko][idx++] = ket_sph_coef(LK, ko, cart_x(S, sc), cart_y(S, sc), cart_z(S, sc));
        }
    }
    return t;
}
template <int LK>
__constant__ KetCoefTable<LK> c_ket_coef = make_ket_table<LK>();

// True when every coefficient of the ket levels below |s| = l_k is exactly
// zero in the tables (spherical kets, l_k <= 4); the kernels then read only the
// top level.
template <int LK>
constexpr bool ket_top_level_only() {
    const KetCoefTable<LK> t = make_ket_table<LK>();
    for (int ko = 0; ko < nsph(LK); ko++)
        for (int i = ncart(LK); i < ket_n_s(LK); i++)
            if (t.v[ko][i] != 0.0) return false;
    return true;
}

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

// E^{0,b}_t along one axis for b <= N, a Gaussian on centre B expanded about
// P: E^{0,b+1}_t = E^{0,b}_{t-1}/(2p) + PB E^{0,b}_t + (t+1) E^{0,b}_{t+1},
// out[b (b+1)/2 + t].
template <int N>
__device__ __forceinline__ void bra_e0b_table(double PB, double inv2p, double* out) {
    double W[N + 1][N + 1];
#pragma unroll
    for (int b = 0; b <= N; b++)
#pragma unroll
        for (int t = 0; t <= N; t++) W[b][t] = 0.0;
    W[0][0] = 1.0;
#pragma unroll
    for (int b = 0; b < N; b++)
#pragma unroll
        for (int t = 0; t <= b + 1; t++) {
            double v = 0.0;
            if (t >= 1) v = inv2p * W[b][t - 1];
            if (t <= b) v = fma(PB, W[b][t], v);
            if (t + 1 <= b) v = fma((double)(t + 1), W[b][t + 1], v);
            W[b + 1][t] = v;
        }
#pragma unroll
    for (int b = 0; b <= N; b++)
#pragma unroll
        for (int t = 0; t <= b; t++) out[b * (b + 1) / 2 + t] = W[b][t];
}

// Fill bra.prim_E (records of e_record<LI, LJ>() doubles per primitive pair):
// one thread per shell pair, looping over its primitive pairs.
template <int LI, int LJ>
__global__ void e_table_kernel(BraTable bra, double* __restrict__ prim_E) {
    constexpr int NE = e_size<LI, LJ>();
    constexpr int NH = e_hrr_size<LI, LJ>();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= bra.n_group) return;
    const double4 AB = bra.grp_AB[g];
    for (int pp = bra.grp_begin[g]; pp < bra.grp_begin[g + 1]; pp++) {
        const double4 PA = bra.prim_PA[pp];
        const double inv2p = 0.5 / bra.prim_P[pp].w;
        double* out = prim_E + (size_t)pp * e_record<LI, LJ>();
        if constexpr (NH > 0) {
            bra_e0b_table<LI + LJ>(PA.x + AB.x, inv2p, out);
            bra_e0b_table<LI + LJ>(PA.y + AB.y, inv2p, out + NH);
            bra_e0b_table<LI + LJ>(PA.z + AB.z, inv2p, out + 2 * NH);
            out += 3 * NH;
        }
        bra_e_table<LI, LJ>(PA.x, AB.x, inv2p, out);
        bra_e_table<LI, LJ>(PA.y, AB.y, inv2p, out + NE);
        bra_e_table<LI, LJ>(PA.z, AB.z, inv2p, out + 2 * NE);
    }
}

// Index of the (0, b) function b = (bx, by, bz) among those with
// LJ <= |b| (order-major, x-major descending within an order).
template <int LJ>
__host__ __device__ constexpr int base_index(int bx, int by, int bz) {
    return herm_index(bx, by, bz) - nherm(LJ - 1);
}

// Cartesian (a, b) block entry, |a| = AX+AY+AZ, from the accumulated (0, b)
// functions by the transfer (a+1_d, b) = (a, b+1_d) - AB_d (a, b).
template <int LJ, int AX, int AY, int AZ, int BX, int BY, int BZ, typename T, typename Acc>
__device__ __forceinline__ T hrr_value(const Acc& acc, int c, T abx, T aby, T abz) {
    if constexpr (AX + AY + AZ == 0) {
        return acc[base_index<LJ>(BX, BY, BZ)][c];
    } else if constexpr (AX > 0) {
        return hrr_value<LJ, AX - 1, AY, AZ, BX + 1, BY, BZ, T>(acc, c, abx, aby, abz) -
               abx * hrr_value<LJ, AX - 1, AY, AZ, BX, BY, BZ, T>(acc, c, abx, aby, abz);
    } else if constexpr (AY > 0) {
        return hrr_value<LJ, AX, AY - 1, AZ, BX, BY + 1, BZ, T>(acc, c, abx, aby, abz) -
               aby * hrr_value<LJ, AX, AY - 1, AZ, BX, BY, BZ, T>(acc, c, abx, aby, abz);
    } else {
        return hrr_value<LJ, AX, AY, AZ - 1, BX, BY, BZ + 1, T>(acc, c, abx, aby, abz) -
               abz * hrr_value<LJ, AX, AY, AZ - 1, BX, BY, BZ, T>(acc, c, abx, aby, abz);
    }
}

// Exponent zeta of the Boys argument and the prefactor of one unit: a primitive
// pair of exponent p and an auxiliary primitive of exponent q, c the product
// of their coefficients (MI/three_center.cpp:46-49 and, for POINT,
// MI/nuclear_attraction.cpp:44-45, 69).  omega == 0 uses one division:
// t = 1/(pq(p+q)), zeta = (pq)^2 t, prefactor = c 2 pi^{5/2} sqrt(p+q) t.
template <int LK, bool POINT>
__device__ __forceinline__ void unit_prefactor(double p, double q, double c, double omega, double& zeta,
                                               double& pref) {
    if constexpr (POINT) {
        static_assert(LK == 0, "point charges have no angular momentum");
        if (omega == 0.0) {
            zeta = p;
            pref = c * 2.0 * kPi / p;
        } else {
            zeta = p * omega * omega / (p + omega * omega);
            pref = c * 2.0 * kPi * omega / (p * sqrt(p + omega * omega));
        }
    } else if (omega == 0.0) {
        const double pq = p * q, s = p + q;
        const double t = 1.0 / (pq * s);
        zeta = pq * pq * t;
        pref = c * kTwoPi52 * sqrt(s) * t;
    } else {
        zeta = 1.0 / (1.0 / p + 1.0 / q + 1.0 / (omega * omega));
        pref = c * kTwoPi52 * omega / (p * q * sqrt(p * q + (p + q) * omega * omega));
    }
    if (LK & 1) pref = -pref;  // (-1)^{|s|} with |s| = LK mod 2
}

// T: arithmetic type of the R tetrahedron, ket, bra and accumulation (double,
// or float for the mixed-precision path).  Boys, R^{(m)}_000, the E^{ij}_t
// recurrences (precomputed in FP64) and the prefactors are FP64 in both.
// POINT: the ket is a unit point charge instead of an auxiliary Gaussian (the
// nuclear-attraction integral V[mu nu C], MI/nuclear_attraction.cpp:23-114):
// zeta = p (omega > 0: p w^2 / (p + w^2)), prefactor c_ab 2 pi / p
// (omega > 0: c_ab 2 pi w / (p sqrt(p + w^2))), l_k = 0.
template <int LI, int LJ, int LK, int V, typename T, bool POINT = false>
__global__ void __launch_bounds__(Fast3c<LI, LJ, LK, V, use_hrr<LI, LJ, T>()>::THREADS,
                                  Fast3c<LI, LJ, LK, V, use_hrr<LI, LJ, T>()>::MIN_CTAS)
k3c_fast(const double* __restrict__ boys_table, BraTable bra, KetTable ket, BatchMap map, double omega,
         double* __restrict__ out, int* __restrict__ work_counter, int total_items) {
    constexpr bool HRR = use_hrr<LI, LJ, T>();
    using C = Fast3c<LI, LJ, LK, V, HRR>;
    static_assert(POINT || ket_top_level_only<LK>(), "spherical ket with lower Hermite levels");
    constexpr int L = C::L;
    constexpr int UB = C::UB;
    constexpr int NU = C::NU;
    // dynamic shared memory (Fast3c::smem_bytes): per block of UB units
    // (primitive pair x auxiliary primitive) the lanes' R^(m)_000 and unit
    // data (CTAs of several warps only), then the R tetrahedron of the current
    // unit, then the units' E tables
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sU = reinterpret_cast<double*>(smem_raw);                   // [UB][NU][32], KS > 1
    T* sR = reinterpret_cast<T*>(sU + (C::KS == 1 ? 0 : UB * NU * 32));  // [NRN][32], entries R0..NR-1
    T* sE = sR + C::NRN * 32;                                           // [UB][3 NE]
    __shared__ int s_item;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    // work_counter[0]: next item; work_counter[1]: status (0 ok, else the
    // first failed self-check: 1 loop bound, 2 molecule/pair index, 3 pair or
    // auxiliary primitive count out of range).
    int* status = work_counter + 1;

    for (int iter = 0;; iter++) {
        if (threadIdx.x == 0) s_item = atomicAdd(work_counter, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= total_items || item < 0) return;
        if (iter > total_items) {  // a CTA can never take more items than exist
            if (threadIdx.x == 0) atomicCAS(status, 0, 1);
            return;
        }

        // molecule of this item: last m with item_begin[m] <= item
        int lo = 0, hi = map.n_mol - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(map.item_begin + mid) <= item) lo = mid;
            else hi = mid - 1;
        }
        const int m = lo;
        const int aux0 = __ldg(map.aux_begin + m);
        const int n_aux = map.aux_count ? __ldg(map.aux_count + m) : __ldg(map.aux_begin + m + 1) - aux0;
        const int n_tiles = (n_aux + 31) >> 5;
        const int local = item - __ldg(map.item_begin + m);
        const int sp_k = local / n_tiles;
        const int tile = local - sp_k * n_tiles;
        int sp = __ldg(map.sp_begin + m) + sp_k, sp_local = sp_k;
        if (map.sp_list) {
            sp = __ldg(map.sp_list + sp);
            sp_local = sp - __ldg(map.sp_first + m);
        }
        const int a_local = tile * 32 + lane;
        const bool valid = a_local < n_aux;
        const int a = aux0 + a_local;

        int kb = 0, nk = 0;
        if (valid) {
            kb = __ldg(ket.grp_begin + a);
            nk = __ldg(ket.grp_begin + a + 1) - kb;
        }
        const int nk_max = __reduce_max_sync(0xffffffffu, nk);
        if (m < 0 || m >= map.n_mol || sp_local < 0 || sp < 0 || sp >= bra.n_group || n_tiles <= 0) {
            if (threadIdx.x == 0) atomicCAS(status, 0, 2);
            continue;  // every value tested here is the same for all threads of the CTA
        }
        const int pb = __ldg(bra.grp_begin + sp), pe = __ldg(bra.grp_begin + sp + 1);
        if (pe < pb || pe - pb > 4096 || nk_max < 0 || nk_max > 4096) {
            if (threadIdx.x == 0) atomicCAS(status, 0, 3);
            continue;
        }

        T acc[C::NB][C::KPW];
#pragma unroll
        for (int i = 0; i < C::NB; i++)
#pragma unroll
            for (int c = 0; c < C::KPW; c++) acc[i][c] = T(0);

        // Units u = (primitive pair, auxiliary primitive) in blocks of UB: the
        // warps first evaluate the units' Boys functions and prefactors in
        // parallel (one warp per unit, no redundancy), then go through the
        // units one by one, splitting each unit's R tetrahedron and ket
        // components between them.
        const int n_units = (pe - pb) * nk_max;
        // One-warp CTAs (KS == 1) keep a unit's values in registers and load
        // the next unit's primitive data and E table while the current unit is
        // evaluated, so a unit's global loads are off its dependency chain;
        // warp barriers replace block barriers.
        constexpr int NE3 = 3 * C::NE;
        constexpr int ERS = e_record<LI, LJ>();
        constexpr bool ONE = C::KS == 1;
        constexpr bool RREG = ONE && C::NRN <= kRRegMax;
        constexpr int EPL = ONE ? (NE3 + 31) / 32 : 1;  // E values per lane
        double4 nP, nC;
        double nca = 0.0, ncc = 0.0, nE[EPL];
        bool nlive = false;
        // units are fetched in order: primitive pair fpp, auxiliary primitive fkk
        int fpp = pb, fkk = 0;
        auto fetch = [&]() {
            nP = bra.prim_P[fpp];
            nca = bra.prim_PA[fpp].w;
            nlive = fkk < nk;
            nC = nlive ? ket.prim_C[kb + fkk] : make_double4(0.0, 0.0, 0.0, 1.0);
            ncc = nlive ? ket.prim_coef[kb + fkk] : 0.0;
#pragma unroll
            for (int r = 0; r < EPL; r++) {
                const int e = lane + 32 * r;
                nE[r] = e < NE3 ? __ldg(bra.prim_E + (size_t)fpp * ERS + C::E_OFF + e) : 0.0;
            }
            if (++fkk == nk_max) {
                fkk = 0;
                fpp++;
            }
        };
        if constexpr (ONE) {
            if (n_units > 0) fetch();
        }
        double uRm[ONE ? L + 1 : 1], uX = 0.0, uY = 0.0, uZ = 0.0, upref = 0.0, uq = 1.0, uinv2q = 0.5;
        for (int u0 = 0; u0 < n_units; u0 += UB) {
            const int nb = n_units - u0 < UB ? n_units - u0 : UB;
            if constexpr (ONE) {
                const double4 P = nP;
                const double4 Cq = nlive ? nC : make_double4(P.x, P.y, P.z, 1.0);
                const double c = nca * ncc;
#pragma unroll
                for (int r = 0; r < EPL; r++)
                    if (lane + 32 * r < NE3) sE[lane + 32 * r] = (T)nE[r];
                if (u0 + 1 < n_units) fetch();
                uX = P.x - Cq.x;
                uY = P.y - Cq.y;
                uZ = P.z - Cq.z;
                // with uncontracted auxiliary shells (nk_max == 1) every unit of
                // the item has the lane's same q
                if (u0 == 0 || nk_max > 1) {
                    uq = Cq.w;
                    uinv2q = 0.5 / uq;
                }
                double zeta;
                unit_prefactor<LK, POINT>(P.w, uq, c, omega, zeta, upref);
                // R^{(m)}_000 = (-2 zeta)^m F_m(zeta |PQ|^2)
                boys<L>(boys_table, zeta * (uX * uX + uY * uY + uZ * uZ), uRm);
                const double f = -2.0 * zeta;
                double g = f;
#pragma unroll
                for (int mm = 1; mm <= L; mm++) {
                    uRm[mm] *= g;
                    g *= f;
                }
            } else {
                for (int e = threadIdx.x; e < nb * NE3; e += C::THREADS) {
                    const int ub = e / NE3, r = e - ub * NE3;
                    const int pp = pb + (nk_max == 1 ? u0 + ub : (u0 + ub) / nk_max);
                    sE[e] = (T)__ldg(bra.prim_E + (size_t)pp * ERS + C::E_OFF + r);
                }
                for (int ub = warp; ub < nb; ub += C::KS) {
                    const int u = u0 + ub;
                    const int up = nk_max == 1 ? u : u / nk_max;  // uncontracted auxiliary shells: no division
                    const int pp = pb + up, kk = u - up * nk_max;
                    const double4 P = bra.prim_P[pp];
                    const double4 PA = bra.prim_PA[pp];
                    const bool live = kk < nk;
                    const double4 Cq = live ? ket.prim_C[kb + kk] : make_double4(P.x, P.y, P.z, 1.0);
                    const double cc = live ? ket.prim_coef[kb + kk] : 0.0;
                    const double q = Cq.w;
                    const double X = P.x - Cq.x, Y = P.y - Cq.y, Z = P.z - Cq.z;
                    double zeta, pref64;
                    unit_prefactor<LK, POINT>(P.w, q, PA.w * cc, omega, zeta, pref64);
                    // R^{(m)}_000 = (-2 zeta)^m F_m(zeta |PQ|^2)
                    double Rm[L + 1];
                    boys<L>(boys_table, zeta * (X * X + Y * Y + Z * Z), Rm);
                    double* unit = sU + ub * NU * 32 + lane;
                    const double f = -2.0 * zeta;
                    double g = 1.0;
#pragma unroll
                    for (int mm = 0; mm <= L; mm++) {
                        unit[mm * 32] = Rm[mm] * g;
                        g *= f;
                    }
                    unit[(L + 1) * 32] = X;
                    unit[(L + 2) * 32] = Y;
                    unit[(L + 3) * 32] = Z;
                    unit[(L + 4) * 32] = pref64;
                    unit[(L + 5) * 32] = q;
                }
                __syncthreads();
            }
            // one-warp CTAs with a small tetrahedron keep it in registers
            // (each lane reads only its own entries): no shared-memory store
            // and load per entry
            T Rr[RREG ? C::NRN : 1];
            // this warp's share of unit ubr's tetrahedron by the closed form
            // (entries are independent), into dst (or Rr)
            auto tetra = [&](int ubr, T* dst) {
                const double* un = sU + ubr * NU * 32 + lane;
                const T Xr = (T)(ONE ? uX : un[(L + 1) * 32]);
                const T Yr = (T)(ONE ? uY : un[(L + 2) * 32]);
                const T Zr = (T)(ONE ? uZ : un[(L + 3) * 32]);
                T Rt[L + 1], px[L + 1], py[L + 1], pz[L + 1];
                px[0] = py[0] = pz[0] = T(1);
#pragma unroll
                for (int mm = 0; mm <= L; mm++) Rt[mm] = (T)(ONE ? uRm[ONE ? mm : 0] : un[mm * 32]);
#pragma unroll
                for (int mm = 1; mm <= L; mm++) {
                    px[mm] = px[mm - 1] * Xr;
                    py[mm] = py[mm - 1] * Yr;
                    pz[mm] = pz[mm - 1] * Zr;
                }
                static_for<0, C::KS>([&](auto g) {
                    constexpr int G = decltype(g)::value;
                    constexpr int lo_e = C::R0 + G * C::RPW;
                    constexpr int hi_e = C::R0 + ((G + 1) * C::RPW < C::NRN ? (G + 1) * C::RPW : C::NRN);
                    if (warp == G) {
                        static_for<lo_e, hi_e>([&](auto e) {
                            constexpr int idx = decltype(e)::value;
                            const T r = r_closed<herm_t(idx), herm_u(idx), herm_v(idx)>(Rt, px, py, pz);
                            if constexpr (RREG) Rr[idx - C::R0] = r;
                            else dst[(idx - C::R0) * 32 + lane] = r;
                        });
                    }
                });
            };
            for (int ub = 0; ub < nb; ub++) {
                const double* unit = sU + ub * NU * 32 + lane;
                const T* sEu = sE + ub * NE3;
                const T pref = (T)(ONE ? upref : unit[(L + 4) * 32]);
                const double q = ONE ? uq : unit[(L + 5) * 32];
                tetra(ub, sR);
                // (1/2q)^{LK - j}: weight of the ket terms with |s| = LK - 2j
                T w[LK / 2 + 1];
                {
                    const double inv2q = ONE ? uinv2q : 0.5 / q;
                    double base = 1.0;
#pragma unroll
                    for (int j = 0; j < LK - LK / 2; j++) base *= inv2q;
#pragma unroll
                    for (int j = LK / 2; j >= 0; j--) {
                        w[j] = (T)base;
                        base *= inv2q;
                    }
                }
                if constexpr (ONE) __syncwarp();
                else __syncthreads();

                // ket + bra.  Warp w owns ket components ko = w * KPW + c, c < KPW.
                // X[c][h] is formed for a set of components first, so that each
                // E^{ij}_t shared-memory load of the bra feeds one FMA per component.
                // bra: acc[ij][c0 + c] += pref * sum_t Ex sum_u Ey sum_v Ez X[c][tuv], c < NC
                auto bra_acc = [&](const auto& X, auto c0_, auto nc_) {
                    constexpr int c0 = decltype(c0_)::value, NC = decltype(nc_)::value;
                    if constexpr (HRR) {
                        // (0, b) functions: acc[b][c0 + c] += pref sum_t E^{0bx}_t sum_u E^{0by}_u
                        // sum_v E^{0bz}_v X[c][tuv], E^{0b}_t at b (b+1)/2 + t per axis
                        static_for<0, C::NB>([&](auto b_) {
                            constexpr int bi = decltype(b_)::value;
                            constexpr int bx = herm_t(nherm(LJ - 1) + bi), by = herm_u(nherm(LJ - 1) + bi),
                                          bz = herm_v(nherm(LJ - 1) + bi);
                            T sxv[NC];
#pragma unroll
                            for (int c = 0; c < NC; c++) sxv[c] = T(0);
                            static_for<0, bx + 1>([&](auto t_) {
                                constexpr int t = decltype(t_)::value;
                                T su[NC];
#pragma unroll
                                for (int c = 0; c < NC; c++) su[c] = T(0);
                                static_for<0, by + 1>([&](auto u_) {
                                    constexpr int u = decltype(u_)::value;
                                    T sv[NC];
#pragma unroll
                                    for (int c = 0; c < NC; c++) sv[c] = T(0);
                                    static_for<0, bz + 1>([&](auto v_) {
                                        constexpr int v = decltype(v_)::value;
                                        const T ez = sEu[2 * C::NE + bz * (bz + 1) / 2 + v];
#pragma unroll
                                        for (int c = 0; c < NC; c++) sv[c] = fma(ez, X[c][herm_index(t, u, v)], sv[c]);
                                    });
                                    const T ey = sEu[C::NE + by * (by + 1) / 2 + u];
#pragma unroll
                                    for (int c = 0; c < NC; c++) su[c] = fma(ey, sv[c], su[c]);
                                });
                                const T ex = sEu[bx * (bx + 1) / 2 + t];
#pragma unroll
                                for (int c = 0; c < NC; c++) sxv[c] = fma(ex, su[c], sxv[c]);
                            });
#pragma unroll
                            for (int c = 0; c < NC; c++) acc[bi][c0 + c] = fma(pref, sxv[c], acc[bi][c0 + c]);
                        });
                    } else
                    static_for<0, C::NI>([&](auto ci_) {
                        constexpr int ci = decltype(ci_)::value;
                        constexpr int ix = cart_x(LI, ci), iy = cart_y(LI, ci), iz = cart_z(LI, ci);
                        static_for<0, C::NJ>([&](auto cj_) {
                            constexpr int cj = decltype(cj_)::value;
                            constexpr int jx = cart_x(LJ, cj), jy = cart_y(LJ, cj), jz = cart_z(LJ, cj);
                            T sxv[NC];
#pragma unroll
                            for (int c = 0; c < NC; c++) sxv[c] = T(0);
                            static_for<0, ix + jx + 1>([&](auto t_) {
                                constexpr int t = decltype(t_)::value;
                                T su[NC];
#pragma unroll
                                for (int c = 0; c < NC; c++) su[c] = T(0);
                                static_for<0, iy + jy + 1>([&](auto u_) {
                                    constexpr int u = decltype(u_)::value;
                                    T sv[NC];
#pragma unroll
                                    for (int c = 0; c < NC; c++) sv[c] = T(0);
                                    static_for<0, iz + jz + 1>([&](auto v_) {
                                        constexpr int v = decltype(v_)::value;
                                        const T ez = sEu[2 * C::NE + e_offset<LJ>(iz, jz) + v];
#pragma unroll
                                        for (int c = 0; c < NC; c++) sv[c] = fma(ez, X[c][herm_index(t, u, v)], sv[c]);
                                    });
                                    const T ey = sEu[C::NE + e_offset<LJ>(iy, jy) + u];
#pragma unroll
                                    for (int c = 0; c < NC; c++) su[c] = fma(ey, sv[c], su[c]);
                                });
                                const T ex = sEu[e_offset<LJ>(ix, jx) + t];
#pragma unroll
                                for (int c = 0; c < NC; c++) sxv[c] = fma(ex, su[c], sxv[c]);
                            });
#pragma unroll
                            for (int c = 0; c < NC; c++)
                                acc[ci * C::NJ + cj][c0 + c] = fma(pref, sxv[c], acc[ci * C::NJ + cj][c0 + c]);
                        });
                    });
                };
                if constexpr (C::KS == 1) {
                    // One warp per CTA (KPW = NKO): ket coefficients are compile-time
                    // constants (zero terms vanish).  When X[KPW][NHB] would hold
                    // more than kXMax values, the components go in chunks (fewer
                    // live registers; an R entry is loaded once per chunk).
                    constexpr int kXMax = variant_xmax(V);
                    constexpr int NCH = (C::KPW * C::NHB + kXMax - 1) / kXMax;
                    constexpr int KCH = (C::KPW + NCH - 1) / NCH;
                    static_for<0, (C::KPW + KCH - 1) / KCH>([&](auto q_) {
                        constexpr int c0 = decltype(q_)::value * KCH;
                        constexpr int NC = C::KPW - c0 < KCH ? C::KPW - c0 : KCH;
                        // keep the compiler from holding the previous chunk's R
                        // values in registers for this one
                        if constexpr (c0 > 0) asm volatile("" ::: "memory");
                        T Xh[NC][C::NHB];
#pragma unroll
                        for (int c = 0; c < NC; c++)
#pragma unroll
                            for (int h = 0; h < C::NHB; h++) Xh[c][h] = T(0);
                        static_for<0, C::NHB>([&](auto h_) {
                            constexpr int h = decltype(h_)::value;
                            constexpr int t = herm_t(h), u = herm_u(h), v = herm_v(h);
                            // top Hermite level |s| = LK only (ket_top_level_only)
                            static_for<0, 1>([&](auto j_) {
                                constexpr int j = decltype(j_)::value;
                                constexpr int S = LK - 2 * j;
                                T part[NC];
#pragma unroll
                                for (int c = 0; c < NC; c++) part[c] = T(0);
                                static_for<0, ncart(S)>([&](auto sc_) {
                                    constexpr int sc = decltype(sc_)::value;
                                    constexpr int sx = cart_x(S, sc), sy = cart_y(S, sc), sz = cart_z(S, sc);
                                    constexpr bool any = [] {
                                        for (int c = c0; c < c0 + NC; c++)
                                            if (ket_sph_coef(LK, c, sx, sy, sz) != 0.0) return true;
                                        return false;
                                    }();
                                    if constexpr (any) {
                                        constexpr int ridx = herm_index(t + sx, u + sy, v + sz) - C::R0;
                                        T r;
                                        if constexpr (RREG) r = Rr[ridx];
                                        else r = sR[ridx * 32 + lane];
                                        static_for<0, NC>([&](auto c_) {
                                            constexpr int c = decltype(c_)::value;
                                            constexpr double kc = ket_sph_coef(LK, c0 + c, sx, sy, sz);
                                            if constexpr (kc != 0.0) part[c] = fma((T)kc, r, part[c]);
                                        });
                                    }
                                });
#pragma unroll
                                for (int c = 0; c < NC; c++) Xh[c][h] = fma(w[j], part[c], Xh[c][h]);
                            });
                        });
                        bra_acc(Xh, ic<c0>{}, ic<NC>{});
                    });
                } else {
                    // Several warps: the same code in every warp, coefficients
                    // from constant memory, so the instruction cache holds one copy.
                    // A warp owning several components forms X for all of them at
                    // once (one tetrahedron load feeds each), or, when that block
                    // would exceed kXMaxMW values, one component at a time.
                    constexpr int kXMaxMW = 24;
                    constexpr int XC = C::KPW * C::NHB > kXMaxMW ? 1 : C::KPW;  // components per X block
                    static_for<0, C::KPW / XC>([&](auto q_) {
                        constexpr int c0 = decltype(q_)::value * XC;
                        if constexpr (c0 > 0) asm volatile("" ::: "memory");
                        T Xh[XC][C::NHB];
#pragma unroll
                        for (int c = 0; c < XC; c++)
#pragma unroll
                            for (int h = 0; h < C::NHB; h++) Xh[c][h] = T(0);
                        int sidx = 0;
                        // top Hermite level |s| = LK only (ket_top_level_only)
                        static_for<0, 1>([&](auto j_) {
                            constexpr int j = decltype(j_)::value;
                            constexpr int S = LK - 2 * j;
                            static_for<0, ncart(S)>([&](auto sc_) {
                                constexpr int sc = decltype(sc_)::value;
                                constexpr int sx = cart_x(S, sc), sy = cart_y(S, sc), sz = cart_z(S, sc);
                                T ce[XC];
                                bool any = false;
#pragma unroll
                                for (int c = 0; c < XC; c++) {
                                    const int ko = warp * C::KPW + c0 + c;
                                    const double cf = ko < C::NKO ? c_ket_coef<LK>.v[ko][sidx + sc] : 0.0;
                                    ce[c] = (T)cf * w[j];
                                    any = any || cf != 0.0;
                                }
                                if (any) {  // warp-uniform
                                    static_for<0, C::NHB>([&](auto h_) {
                                        constexpr int h = decltype(h_)::value;
                                        constexpr int t = herm_t(h), u = herm_u(h), v = herm_v(h);
                                        const T r = sR[(herm_index(t + sx, u + sy, v + sz) - C::R0) * 32 + lane];
#pragma unroll
                                        for (int c = 0; c < XC; c++) Xh[c][h] = fma(ce[c], r, Xh[c][h]);
                                    });
                                }
                            });
                            sidx += ncart(S);
                        });
                        bra_acc(Xh, ic<c0>{}, ic<XC>{});
                    });
                }
                if constexpr (ONE) __syncwarp();
                else __syncthreads();
            }
        }

        // Epilogue: (transfer l_i onto A,) bra Cartesian -> spherical, coalesced
        // packed stores.
        const size_t obase = (size_t)__ldg(map.out_begin + m);
        double wsum = 0.0;
        T abx = T(0), aby = T(0), abz = T(0);
        if constexpr (HRR) {
            const double4 AB = bra.grp_AB[sp];
            abx = (T)AB.x;
            aby = (T)AB.y;
            abz = (T)AB.z;
        }
        static_for<0, C::KPW>([&](auto c_) {
            constexpr int c = decltype(c_)::value;
            const int ko = warp * C::KPW + c;
            if (ko < C::NKO) {
                // Cartesian (i, j) entry of ket component c
                auto cart_ij = [&](auto ci_, auto cj_) -> T {
                    constexpr int ci = decltype(ci_)::value, cj = decltype(cj_)::value;
                    if constexpr (HRR)
                        return hrr_value<LJ, cart_x(LI, ci), cart_y(LI, ci), cart_z(LI, ci), cart_x(LJ, cj),
                                         cart_y(LJ, cj), cart_z(LJ, cj), T>(acc, c, abx, aby, abz);
                    else
                        return acc[ci * C::NJ + cj][c];
                };
                static_for<0, nsph(LI)>([&](auto I_) {
                    constexpr int I = decltype(I_)::value;
                    static_for<0, nsph(LJ)>([&](auto J_) {
                        constexpr int J = decltype(J_)::value;
                        T v = T(0);
                        static_for<0, C::NI>([&](auto ci_) {
                            constexpr int ci = decltype(ci_)::value;
                            constexpr double wi = sph_coef(LI, I, ci);
                            if constexpr (wi != 0.0) {
                                T vj = T(0);
                                static_for<0, C::NJ>([&](auto cj_) {
                                    constexpr int cj = decltype(cj_)::value;
                                    constexpr double wj = sph_coef(LJ, J, cj);
                                    if constexpr (wj != 0.0) vj = fma((T)wj, cart_ij(ci_, cj_), vj);
                                });
                                v = fma((T)wi, vj, v);
                            }
                        });
                        if (valid) {
                            const size_t row = ((size_t)sp_local * C::NIJS + I * nsph(LJ) + J) * C::NKO + ko;
                            out[obase + row * n_aux + a_local] = (double)v;
                            wsum += (double)v;
                        }
                    });
                });
            }
        });
        if (map.checksum) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
            if (lane == 0) atomicAdd(map.checksum + m, wsum);
        }
    }
}

// Occupancy-sized persistent grid for one class (per device: the shared-memory
// attribute and the occupancy are set up on each device's first launch).
template <int LI, int LJ, int LK, int V, typename T, bool POINT = false>
static int launch_one(const double* boys_table, const BraTable& bra, const KetTable& ket, const BatchMap& map,
                      int total_items, double omega, double* out, int* counter, cudaStream_t s) {
    using C = Fast3c<LI, LJ, LK, V, use_hrr<LI, LJ, T>()>;
    if (total_items <= 0) return 0;
    constexpr size_t smem = C::template smem_bytes<T>();
    static std::atomic<int> max_blocks[kMaxDevices];
    const int grid = persistent_grid(reinterpret_cast<const void*>(k3c_fast<LI, LJ, LK, V, T, POINT>), C::THREADS,
                                     smem, max_blocks);
    if (grid <= 0) return 2;
    const int blocks = total_items < grid ? total_items : grid;
    k3c_fast<LI, LJ, LK, V, T, POINT><<<blocks, C::THREADS, smem, s>>>(boys_table, bra, ket, map, omega, out,
                                                                       counter, total_items);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

template <int LI, int LJ>
static int launch_e_table(const BraTable& bra, double* prim_E, cudaStream_t s) {
    if (bra.n_group == 0) return 0;
    e_table_kernel<LI, LJ><<<(bra.n_group + 127) / 128, 128, 0, s>>>(bra, prim_E);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace eip
