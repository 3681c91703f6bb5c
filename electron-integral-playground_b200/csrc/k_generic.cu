// General kernels: every angular class the C ABI accepts, with run-time
// angular momenta (orbital l <= 6, auxiliary l <= 9; reference
// c_library/angular.h:3-4), over the same multi-molecule work list as the fast
// kernels.  They carry what the fast templated kernels do not: Cartesian
// output, (mu nu|P) classes beyond d-d|g, the high-l metric and
// nuclear-attraction classes.
//
// general_kernel: persistent CTAs of kGenThreads threads; one work item is
// one contracted block (shell pair, auxiliary shell or point charge, chunk of
// ket components), computed as
//   (mu nu|P) = sum_{prim pairs} sum_{aux prims} pref
//               sum_{tuv} E^{ij}_{tuv} sum_s (-1)^{|s|} E^{k}_s R_{t+s_x,u+s_y,v+s_z}
// with the two-centre coefficients E^{ij}_t built per primitive pair in FP64
// (vertical recursion on centre A, then the transfer to centre B,
// c_library/mcmurchie_davidson_E_term.hpp:22-45, 166-199).  Per block of
// kGenUB units (primitive pair x auxiliary primitive) the CTA first evaluates,
// one thread per unit, the prefactor, Boys function, scaled R^{(m)}_000 and
// coordinate powers, and per unit and axis the E^{ij}_t table (or, in a
// batch, copies it from the table precomputed per primitive pair by
// general_e_table_kernel); then, unit by unit, all threads split (1) the
// Hermite tetrahedron R_{tuv} (closed form), (2) the ket contraction X[h][k]
// (stored v-innermost, spherical kets through compact lists of their non-zero
// terms), (3) the bra contraction into accumulators held in registers
// (kGenAcc per thread; the bra pairs ranked by their loop shape so that a
// warp's lanes run the same trip counts).  Blocks with many units are split
// into several items whose partial blocks the last to arrive adds up.  (Transferring after the
// contraction instead, as the fast FP64 kernels do for l <= 2, loses up to
// 1e-9 to cancellation for g-g pairs with distant centres and extreme
// exponents, so the high-l classes transfer per primitive pair.)
//
// Spherical kets use only the top Hermite level |s| = l_k: a real solid
// harmonic is a harmonic polynomial, so its Gaussian's Hermite expansion has
// no lower terms (Hobson's theorem), and the coefficient of s on that level is
// the spherical coefficient of the Cartesian component s itself.  Cartesian
// kets use every level with the one-centre coefficients
// (c_library/mcmurchie_davidson_E_term.hpp:132-139).
//
// Prefactors: Coulomb 2 pi^{5/2} / (p q sqrt(p+q)) (MI/three_center.cpp:46-49,
// MI/two_center.cpp:34-37; erf-attenuated for omega > 0); point charges
// 2 pi / p with zeta = p (MI/nuclear_attraction.cpp:44-45, :69).
//
// Output: the packed layout of the fast kernels, molecule m's block at
// out_begin[m]:
//   out[((pair * n_io * n_jo + I * n_jo + J) * n_ko + K) * n_aux_m + aux]
// (spherical or per-component-normalised Cartesian components).
//
// overlap_raw_kernel / transform_kernel: the overlap S (E-only).
#include <algorithm>
#include <mutex>

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

// Index of (x, y, z) among the Cartesian components of l = x + y + z.
__host__ __device__ __forceinline__ int cart_index(int x, int y, int z) {
    const int l = x + y + z;
    return (l - x) * (l - x + 1) / 2 + z;
}

// Hermite index of (t, u, v) in the order-major tetrahedron (herm_index, run time).
__device__ __forceinline__ int herm_idx(int t, int u, int v) {
    const int N = t + u + v;
    return N * (N + 1) * (N + 2) / 6 + cart_index(t, u, v);
}

constexpr int kGenThreads = 128;
constexpr int kGenAcc = 16;   // bra accumulators per thread
constexpr int kGenUB = 4;     // units per block
constexpr int kGenMaxL = 21;  // 6 + 6 + 9
constexpr size_t kGenMaxSmem = 200 * 1024;
constexpr int kGenMaxSplits = 64;

// Shape of one class for the general kernel, computed on the host.
struct GenShape {
    int li, lj, lk, lij, L;
    int point, spherical;
    int nij;        // Cartesian (i, j) pairs of the bra
    int nhb;        // bra Hermite entries, t + u + v <= l_i + l_j
    int n_io, n_jo, n_ko;
    int nkc;        // Cartesian components of l_k
    int ko_chunk, n_chunks;
    int n_splits;   // items per block and chunk, each over a share of the units (set per launch)
    int nea;        // E^{ij}_t entries per axis: (l_i+1)(l_j+1)(l_i+l_j+1)
    int rmin;       // lowest Hermite order of R the ket reads
    int nr;         // nherm(L)
    int unit_dbl;   // doubles per unit record
    // shared-memory offsets, in doubles
    int o_unit, o_hr, o_ket, o_kc, o_dec, o_row, o_ij, o_work, o_x, o_base;
    int smem_dbl;
};

// E^{ij}_t along one axis for every i <= l_i, j <= l_j, at E[(i (l_j+1) + j)(l_i+l_j+1) + t]:
// E^{i+1,0}_t = E^{i,0}_{t-1} / (2p) + PA E^{i,0}_t + (t+1) E^{i,0}_{t+1} for
// i < l_i + l_j, then E^{i,j+1}_t = E^{i+1,j}_t + AB E^{i,j}_t, level j kept in
// W (rows i <= l_i + l_j - j) and rows i <= l_i stored
// (c_library/mcmurchie_davidson_E_term.hpp:22-45, 166-199).
__device__ void general_e_axis(int li, int lj, double pa_d, double ab_d, double inv2p, double* E) {
    const int N = li + lj, T1 = li + lj + 1;
    double W[kMaxOrbitalL * 2 + 1][kMaxOrbitalL * 2 + 1];
    for (int i = 0; i <= N; i++)
        for (int t = 0; t <= N; t++) W[i][t] = 0.0;
    W[0][0] = 1.0;
    for (int i = 0; i < N; i++)
        for (int t = 0; t <= i + 1; t++) {
            double v = 0.0;
            if (t >= 1) v = inv2p * W[i][t - 1];
            if (t <= i) v = fma(pa_d, W[i][t], v);
            if (t + 1 <= i) v = fma((double)(t + 1), W[i][t + 1], v);
            W[i + 1][t] = v;
        }
    for (int j = 0; j <= lj; j++) {
        for (int i = 0; i <= li; i++)
            for (int t = 0; t <= N; t++) E[(i * (lj + 1) + j) * T1 + t] = W[i][t];
        if (j == lj) break;
        for (int i = 0; i + j + 1 <= N; i++)
            for (int t = 0; t <= N; t++) W[i][t] = fma(ab_d, W[i][t], W[i + 1][t]);
    }
}

// Unit record: [0, L] R^{(m)}_000 (-2 zeta)^m; L+1 prefactor; then X, Y, Z
// powers (L+1 each); then E^{ij}_t for x, y, z (nea each, index
// (i (l_j+1) + j)(l_i+l_j+1) + t); then, Cartesian
// kets only, the signed one-centre coefficients (l_k+1)^2.
__host__ __device__ inline int unit_pow(const GenShape& g) { return g.L + 2; }
__host__ __device__ inline int unit_e(const GenShape& g) { return g.L + 2 + 3 * (g.L + 1); }
__host__ __device__ inline int unit_ek(const GenShape& g) { return unit_e(g) + 3 * g.nea; }

static GenShape general_shape(int li, int lj, int lk, bool point, bool spherical) {
    GenShape g{};
    g.li = li; g.lj = lj; g.lk = point ? 0 : lk; g.lij = li + lj; g.L = g.lij + g.lk;
    g.point = point; g.spherical = spherical;
    g.nij = ncart(li) * ncart(lj);
    g.nhb = nherm(g.lij);
    g.n_io = spherical ? nsph(li) : ncart(li);
    g.n_jo = spherical ? nsph(lj) : ncart(lj);
    g.n_ko = point ? 1 : (spherical ? nsph(g.lk) : ncart(g.lk));
    g.nkc = ncart(g.lk);
    g.ko_chunk = std::max(1, std::min(g.n_ko, kGenThreads * kGenAcc / g.nij));
    g.n_chunks = (g.n_ko + g.ko_chunk - 1) / g.ko_chunk;
    g.n_splits = 1;
    g.nea = (li + 1) * (lj + 1) * (g.lij + 1);
    g.rmin = (spherical && !point) ? g.lk : 0;
    g.nr = nherm(g.L);
    g.unit_dbl = unit_ek(g) + ((!spherical && !point) ? (g.lk + 1) * (g.lk + 1) : 0);
    // layout: closed-form coefficients (first: the same place for every class
    // of a launch) | unit block | ket rows | tetrahedron decode (ints) | work
    // region: [R | X] during the unit loop, the accumulated Cartesian block in
    // the epilogue
    int o = 0;
    g.o_hr = o; o += (kGenMaxL + 1) * (kGenMaxL + 1);
    g.o_unit = o; o += kGenUB * g.unit_dbl;
    g.o_ket = o; o += g.n_ko * g.nkc;
    g.o_kc = o; o += (g.n_ko * g.nkc + g.n_ko + 1) / 2;
    g.o_dec = o; o += (g.nr + 1) / 2;
    g.o_row = o; o += ((g.lij + 1) * (g.lij + 1) + 1) / 2;
    g.o_ij = o; o += (g.nij + 1) / 2;
    g.o_work = o;
    g.o_x = o + g.nr;
    g.o_base = o;
    const int loop_end = g.o_x + g.nhb * g.ko_chunk;
    const int epi_end = g.o_base + g.nij * g.ko_chunk;
    g.smem_dbl = std::max(loop_end, epi_end);
    return g;
}

// One class of a general launch: its shape, tables and work map; status is
// its self-check word (0 ok, else the first failed check: 1 loop bound,
// 2 molecule/pair/auxiliary index, 3 count).
struct GenClassDesc {
    GenShape g;
    BraTable bra;
    KetTable ket;
    BatchMap map;
    int* status;
    const double* etab;  // optional: E tables per primitive pair (general_e_table_kernel)
    double* partial;  // split items: partial blocks, nij * ko_chunk doubles per item
    int* arrive;      // split items: arrivals per block and chunk
};

// Up to kGenMaxClasses classes in one launch, passed by value in the kernel's
// parameter space (about 27 KB of the 32 KB it may hold): every CTA reads the
// descriptor of its current item's class from there.  Items of class c are
// numbered from item0[c].  96 covers every (l_i <= l_j <= 4 | l_k <= 5) class.
constexpr int kGenMaxClasses = 96;
struct GenLaunch {
    int n_classes;
    int item0[kGenMaxClasses + 1];
    GenClassDesc cls[kGenMaxClasses];
};
static_assert(sizeof(GenLaunch) + 64 <= 32764, "general launch descriptors exceed the kernel parameter space");

__global__ void __launch_bounds__(kGenThreads)
general_kernel(const double* __restrict__ boys_table, const __grid_constant__ GenLaunch lp,
               const int2* __restrict__ perm, double omega, double* __restrict__ out, int* __restrict__ work_counter,
               int total_items) {
    extern __shared__ __align__(16) double gsm[];
    __shared__ int s_item, s_last;
    const int tid = threadIdx.x;

    // per-CTA table shared by every class: closed-form Hermite coefficients
    // (first in every class's layout)
    {
        double* sHR = gsm;
        for (int e = tid; e < (kGenMaxL + 1) * (kGenMaxL + 1); e += kGenThreads) {
            const int t = e / (kGenMaxL + 1), m = e % (kGenMaxL + 1);
            double r = 0.0;
            if (m >= (t + 1) / 2 && m <= t) {
                r = 1.0;
                for (int i = 2; i <= t; i++) r *= i;
                for (int i = 2; i <= 2 * m - t; i++) r /= i;
                for (int i = 2; i <= t - m; i++) r /= i;
                for (int i = 0; i < t - m; i++) r *= 0.5;
            }
            sHR[e] = r;
        }
    }
    int cur = -1;  // class whose per-class tables are in shared memory

    for (int iter = 0;; iter++) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(work_counter, 1);
        __syncthreads();
        const int gitem = s_item;
        if (gitem >= total_items || gitem < 0) return;
        // the class of this item and its number within the class (the same
        // for all threads of the CTA)
        int c, item;
        if (perm) {
            const int2 pc = __ldg(perm + gitem);
            c = pc.x;
            item = pc.y;
        } else {
            int lo = 0, hi = lp.n_classes - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (lp.item0[mid] <= gitem) lo = mid;
                else hi = mid - 1;
            }
            c = lo;
            item = gitem - lp.item0[c];
        }
        if (c < 0 || c >= lp.n_classes) {
            if (tid == 0) atomicCAS(lp.cls[0].status, 0, 2);
            continue;
        }
        const GenShape& g = lp.cls[c].g;
        const BraTable& bra = lp.cls[c].bra;
        const KetTable& ket = lp.cls[c].ket;
        const BatchMap& map = lp.cls[c].map;
        int* status = lp.cls[c].status;
        if (iter > total_items) {  // a CTA can never take more items than exist
            if (tid == 0) atomicCAS(status, 0, 1);
            return;
        }
        double* sUnit = gsm + g.o_unit;
        const double* sHR = gsm + g.o_hr;
        // spherical kets: per component ko its n = sKn[ko] non-zero top-level
        // terms, weight sKet[ko nkc + j] and code sKc[ko nkc + j] = (l_k - s_x) | s_z << 8
        double* sKet = gsm + g.o_ket;
        int* sKc = reinterpret_cast<int*>(gsm + g.o_kc);
        int* sKn = sKc + g.n_ko * g.nkc;
        int* sDec = reinterpret_cast<int*>(gsm + g.o_dec);
        // X is stored with v innermost: entry (t, u, v) at sRow[t (l_i+l_j+1) + u] + v
        int* sRow = reinterpret_cast<int*>(gsm + g.o_row);
        // bra pairs in the order of their (i_x+j_x, i_y+j_y, i_z+j_z): sIJ[r] is the pair at rank r
        int* sIJ = reinterpret_cast<int*>(gsm + g.o_ij);
        double* sR = gsm + g.o_work;
        double* sX = gsm + g.o_x;
        double* sBase = gsm + g.o_base;
        if (c != cur) {
            // per-class tables: spherical ket rows, tetrahedron decode (t | u << 8 | v << 16)
            if (g.spherical && !g.point)
                for (int ko = tid; ko < g.n_ko; ko += kGenThreads) {
                    int n = 0;
                    for (int ck = 0; ck < g.nkc; ck++) {
                        const double w = c_sph_coef[c_sph_offset[g.lk] + ko * g.nkc + ck];
                        if (w == 0.0) continue;
                        int sx, sy, sz;
                        cart_decode(g.lk, ck, sx, sy, sz);
                        sKet[ko * g.nkc + n] = w;
                        sKc[ko * g.nkc + n] = (g.lk - sx) | (sz << 8);
                        n++;
                    }
                    sKn[ko] = n;
                }
            for (int N = 0; N <= g.L; N++)
                for (int k = tid; k < ncart(N); k += kGenThreads) {
                    int x, y, z;
                    cart_decode(N, k, x, y, z);
                    sDec[nherm(N - 1) + k] = x | (y << 8) | (z << 16);
                }
            {
                const int T1 = g.lij + 1;
                for (int e = tid; e < T1 * T1; e += kGenThreads) {
                    const int t = e / T1, u = e - t * T1;
                    int pos = -1;
                    if (t + u <= g.lij) {
                        pos = 0;
                        for (int tt = 0; tt < t; tt++) pos += (g.lij - tt + 1) * (g.lij - tt + 2) / 2;
                        for (int uu = 0; uu < u; uu++) pos += g.lij - t - uu + 1;
                    }
                    sRow[e] = pos;
                }
            }
            __syncthreads();
            {
                // The bra loops over t <= i_x+j_x, u <= i_y+j_y, v <= i_z+j_z;
                // ranking the pairs by that triple gives the lanes of a warp
                // (consecutive accumulator entries) mostly the same loop shape.
                int* sKey = reinterpret_cast<int*>(gsm + g.o_work);  // free between items
                const int nj_c = ncart(g.lj);
                for (int ij = tid; ij < g.nij; ij += kGenThreads) {
                    const int ci = ij / nj_c, cj = ij - ci * nj_c;
                    const int da = sDec[nherm(g.li - 1) + ci], db = sDec[nherm(g.lj - 1) + cj];
                    const int sx = (da & 255) + (db & 255), sy = ((da >> 8) & 255) + ((db >> 8) & 255),
                              sz = (da >> 16) + (db >> 16);
                    sKey[ij] = (sx * 32 + sy) * 32 + sz;
                }
                __syncthreads();
                for (int ij = tid; ij < g.nij; ij += kGenThreads) {
                    const int key = sKey[ij];
                    int r = 0;
                    for (int o = 0; o < g.nij; o++) {
                        const int ok = sKey[o];
                        r += (ok < key) || (ok == key && o < ij);
                    }
                    sIJ[r] = ij;
                }
            }
            cur = c;
            __syncthreads();
        }
        // accumulator entry e = tid + kGenThreads * k holds (Cartesian pair ij, ket component)
        const int n_ent = g.nij * g.ko_chunk;
        int lo = 0, hi = map.n_mol - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(map.item_begin + mid) <= item) lo = mid;
            else hi = mid - 1;
        }
        const int m = lo;
        const int aux0 = __ldg(map.aux_begin + m);
        const int n_aux = map.aux_count ? __ldg(map.aux_count + m) : __ldg(map.aux_begin + m + 1) - aux0;
        const int local = item - __ldg(map.item_begin + m);
        // local = ((pair * n_aux + aux) * n_chunks + chunk) * n_splits + split
        const int split = local % g.n_splits;
        const int chunk = (local / g.n_splits) % g.n_chunks;
        const int rest = local / (g.n_splits * g.n_chunks);
        const int a_local = n_aux > 0 ? rest % n_aux : 0;
        const int sp_k = n_aux > 0 ? rest / n_aux : 0;
        const int sp = __ldg(map.sp_begin + m) + sp_k;
        const int a = aux0 + a_local;
        // every value tested here is the same for all threads of the CTA
        if (n_aux <= 0 || sp < 0 || sp >= bra.n_group || sp >= __ldg(map.sp_begin + m + 1) || a < 0 ||
            a >= ket.n_group) {
            if (tid == 0) atomicCAS(status, 0, 2);
            continue;
        }
        const int pb = __ldg(bra.grp_begin + sp), pe = __ldg(bra.grp_begin + sp + 1);
        const int kb = __ldg(ket.grp_begin + a), ke = __ldg(ket.grp_begin + a + 1);
        const int npp = pe - pb, nkp = ke - kb;
        if (npp < 0 || npp > 4096 || nkp < 0 || nkp > 4096) {
            if (tid == 0) atomicCAS(status, 0, 3);
            continue;
        }
        const double4 AB = bra.grp_AB[sp];
        const double* etab = lp.cls[c].etab;  // per primitive pair E tables, or computed here
        const int ko0 = chunk * g.ko_chunk;
        const int nkoc = min(g.ko_chunk, g.n_ko - ko0);

        double acc[kGenAcc];
#pragma unroll
        for (int k = 0; k < kGenAcc; k++) acc[k] = 0.0;

        // this item's units: its split's share of the block's
        const int n_all = npp * nkp;
        const int u_begin = (int)((long long)n_all * split / g.n_splits);
        const int n_units = (int)((long long)n_all * (split + 1) / g.n_splits);
        for (int u0 = u_begin; u0 < n_units; u0 += kGenUB) {
            const int nb = min(kGenUB, n_units - u0);
            __syncthreads();  // the previous block's unit records are no longer read
            // (A) per unit: prefactor, Boys, R^{(m)}_000, powers; per unit and axis: E^{0 b}_t
            for (int w = tid; w < (etab ? nb : 4 * nb); w += kGenThreads) {
                const int ub = w < nb ? w : (w - nb) / 3;
                const int u = u0 + ub;
                const int pp = pb + u / nkp, kp = kb + u % nkp;
                double* U = sUnit + ub * g.unit_dbl;
                const double4 P = bra.prim_P[pp];
                if (w < nb) {
                    const double4 PA = bra.prim_PA[pp];
                    const double4 Cq = ket.prim_C[kp];
                    const double c = PA.w * ket.prim_coef[kp];
                    const double p = P.w, q = Cq.w;
                    double zeta, pref;
                    if (g.point) {
                        if (omega == 0.0) {
                            zeta = p;
                            pref = c * 2.0 * kPi / p;
                        } else {
                            zeta = p * omega * omega / (p + omega * omega);
                            pref = c * 2.0 * kPi * omega / (p * sqrt(p + omega * omega));
                        }
                    } else {
                        if (omega == 0.0) {
                            zeta = p * q / (p + q);
                            pref = c * kTwoPi52 / (p * q * sqrt(p + q));
                        } else {
                            zeta = 1.0 / (1.0 / p + 1.0 / q + 1.0 / (omega * omega));
                            pref = c * kTwoPi52 * omega / (p * q * sqrt(p * q + (p + q) * omega * omega));
                        }
                    }
                    const double X = P.x - Cq.x, Y = P.y - Cq.y, Z = P.z - Cq.z;
                    double F[kMaxBoysM + 1];
                    boys_rt(boys_table, g.L, zeta * (X * X + Y * Y + Z * Z), F);
                    double f = 1.0;
                    for (int mm = 0; mm <= g.L; mm++) {
                        U[mm] = F[mm] * f;
                        f *= -2.0 * zeta;
                    }
                    if (g.spherical && !g.point) {
                        // top Hermite level only: weight (-1/(2q))^{l_k}
                        const double w2q = -0.5 / q;
                        for (int i = 0; i < g.lk; i++) pref *= w2q;
                    } else if (!g.point) {
                        // signed one-centre coefficients (-1)^s E^{k,0}_s(q)
                        double* ek = U + unit_ek(g);
                        const double inv2q = 0.5 / q;
                        for (int k = 0; k <= g.lk; k++)
                            for (int s = 0; s <= g.lk; s++) {
                                double cf = 0.0;
                                if (s <= k && !((k - s) & 1)) {
                                    const int h = (k - s) / 2;
                                    cf = 1.0;
                                    for (int i = 2; i <= k; i++) cf *= i;
                                    for (int i = 2; i <= h; i++) cf /= i;
                                    for (int i = 2; i <= s; i++) cf /= i;
                                    for (int i = 0; i < h; i++) cf *= 0.5;
                                    for (int i = 0; i < (k + s) / 2; i++) cf *= inv2q;
                                    if (s & 1) cf = -cf;
                                }
                                ek[k * (g.lk + 1) + s] = cf;
                            }
                    }
                    U[g.L + 1] = pref;
                    double* pw = U + unit_pow(g);
                    double px = 1.0, py = 1.0, pz = 1.0;
                    for (int k = 0; k <= g.L; k++) {
                        pw[k] = px;
                        pw[g.L + 1 + k] = py;
                        pw[2 * (g.L + 1) + k] = pz;
                        px *= X;
                        py *= Y;
                        pz *= Z;
                    }
                } else {
                    const int d = (w - nb) % 3;
                    const double4 PA = bra.prim_PA[pp];
                    const double pa_d = d == 0 ? PA.x : (d == 1 ? PA.y : PA.z);
                    const double ab_d = d == 0 ? AB.x : (d == 1 ? AB.y : AB.z);
                    general_e_axis(g.li, g.lj, pa_d, ab_d, 0.5 / P.w, U + unit_e(g) + d * g.nea);
                }
            }
            if (etab) {
                // the units' E tables, precomputed per primitive pair: a coalesced copy
                const int ne3 = 3 * g.nea;
                for (int e = tid; e < nb * ne3; e += kGenThreads) {
                    const int ub = e / ne3, r = e - ub * ne3;
                    const int pp = pb + (u0 + ub) / nkp;
                    sUnit[ub * g.unit_dbl + unit_e(g) + r] = __ldg(etab + (size_t)pp * ne3 + r);
                }
            }
            __syncthreads();
            for (int ub = 0; ub < nb; ub++) {
                const double* U = sUnit + ub * g.unit_dbl;
                // (1) tetrahedron entries of order >= rmin, closed form
                // (c_library/mcmurchie_davidson_R_term.hpp:31-37)
                {
                    const double* Rm = U;
                    const double* px = U + unit_pow(g);
                    const double* py = px + g.L + 1;
                    const double* pz = py + g.L + 1;
                    for (int idx = nherm(g.rmin - 1) + tid; idx < g.nr; idx += kGenThreads) {
                        const int dc = sDec[idx];
                        const int t = dc & 255, u = (dc >> 8) & 255, v = dc >> 16;
                        double r = 0.0;
                        for (int mx = (t + 1) / 2; mx <= t; mx++) {
                            double ry = 0.0;
                            for (int my = (u + 1) / 2; my <= u; my++) {
                                double rz = 0.0;
                                for (int mz = (v + 1) / 2; mz <= v; mz++)
                                    rz = fma(sHR[v * (kGenMaxL + 1) + mz] * pz[2 * mz - v], Rm[mx + my + mz], rz);
                                ry = fma(sHR[u * (kGenMaxL + 1) + my] * py[2 * my - u], rz, ry);
                            }
                            r = fma(sHR[t * (kGenMaxL + 1) + mx] * px[2 * mx - t], ry, r);
                        }
                        sR[idx] = r;
                    }
                }
                __syncthreads();
                // (2) ket: X[h][k] for the chunk's ket components
                for (int e = tid; e < g.nhb * nkoc; e += kGenThreads) {
                    const int h = e / nkoc, kl = e - h * nkoc, ko = ko0 + kl;
                    const int dh = sDec[h];
                    const int t = dh & 255, u = (dh >> 8) & 255, v = dh >> 16;
                    double x = 0.0;
                    if (g.point) {
                        x = sR[h];
                    } else if (g.spherical) {
                        // R index of h + s, |s| = l_k: order N = |h| + l_k, so
                        // herm_idx = nherm(N-1) + m (m+1) / 2 + v + s_z with
                        // m = N - (t + s_x) = u + v + l_k - s_x
                        const double* w = sKet + ko * g.nkc;
                        const int* code = sKc + ko * g.nkc;
                        const int N = t + u + v + g.lk;
                        const int base = N * (N + 1) * (N + 2) / 6 + v, q = u + v;
                        for (int j = 0; j < sKn[ko]; j++) {
                            const int cd = code[j];
                            const int mm = q + (cd & 255);
                            x = fma(w[j], sR[base + ((mm * (mm + 1)) >> 1) + (cd >> 8)], x);
                        }
                    } else {
                        int kx, ky, kz;
                        cart_decode(g.lk, ko, kx, ky, kz);
                        const double* ek = U + unit_ek(g);
                        const int w1 = g.lk + 1;
                        for (int sx = kx & 1; sx <= kx; sx += 2)
                            for (int sy = ky & 1; sy <= ky; sy += 2) {
                                const double exy = ek[kx * w1 + sx] * ek[ky * w1 + sy];
                                for (int sz = kz & 1; sz <= kz; sz += 2)
                                    x = fma(exy * ek[kz * w1 + sz], sR[herm_idx(t + sx, u + sy, v + sz)], x);
                            }
                    }
                    sX[(sRow[t * (g.lij + 1) + u] + v) * nkoc + kl] = x;
                }
                __syncthreads();
                // (3) bra: acc[(ij, k)] += pref sum_t Ex sum_u Ey sum_v Ez X[tuv][k]
                {
                    const double pref = U[g.L + 1];
                    const double* Ex = U + unit_e(g);
                    const double* Ey = Ex + g.nea;
                    const double* Ez = Ey + g.nea;
#pragma unroll
                    for (int k = 0; k < kGenAcc; k++) {
                        const int e = tid + kGenThreads * k;
                        if (e < n_ent) {
                            const int rk = e / g.ko_chunk, kl = e - rk * g.ko_chunk;
                            const int ij = sIJ[rk];
                            if (kl < nkoc) {
                                const int ci = ij / ncart(g.lj), cj = ij - ci * ncart(g.lj);
                                const int da = sDec[nherm(g.li - 1) + ci], db = sDec[nherm(g.lj - 1) + cj];
                                const int ix = da & 255, iy = (da >> 8) & 255, iz = da >> 16;
                                const int jx = db & 255, jy = (db >> 8) & 255, jz = db >> 16;
                                const int T1 = g.lij + 1, J1 = g.lj + 1;
                                const double* ex = Ex + (ix * J1 + jx) * T1;
                                const double* ey = Ey + (iy * J1 + jy) * T1;
                                const double* ez = Ez + (iz * J1 + jz) * T1;
                                double s = 0.0;
                                for (int t = 0; t <= ix + jx; t++) {
                                    double su = 0.0;
                                    const int* row = sRow + t * T1;
                                    for (int u = 0; u <= iy + jy; u++) {
                                        double sv = 0.0;
                                        const double* xv = sX + row[u] * nkoc + kl;
                                        for (int v = 0; v <= iz + jz; v++) sv = fma(ez[v], xv[v * nkoc], sv);
                                        su = fma(ey[u], sv, su);
                                    }
                                    s = fma(ex[t], su, s);
                                }
                                acc[k] = fma(pref, s, acc[k]);
                            }
                        }
                    }
                }
            }
        }
        if (g.n_splits > 1) {
            // Split block: write this share, count the arrival; the last split
            // to arrive adds the shares in split order (the same sum whichever
            // CTA is last) and goes on to the epilogue, the others take their
            // next item.
            double* part = lp.cls[c].partial + (size_t)item * n_ent;
#pragma unroll
            for (int k = 0; k < kGenAcc; k++) {
                const int e = tid + kGenThreads * k;
                if (e < n_ent) part[e] = acc[k];
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) s_last = atomicAdd(lp.cls[c].arrive + item / g.n_splits, 1) == g.n_splits - 1;
            __syncthreads();
            if (!s_last) continue;
            __threadfence();
            const double* first = lp.cls[c].partial + (size_t)(item - split) * n_ent;
#pragma unroll
            for (int k = 0; k < kGenAcc; k++) {
                const int e = tid + kGenThreads * k;
                double v = 0.0;
                if (e < n_ent)
                    for (int q = 0; q < g.n_splits; q++) v += __ldcg(first + (size_t)q * n_ent + e);
                acc[k] = v;
            }
            if (tid == 0) lp.cls[c].arrive[item / g.n_splits] = 0;  // ready for the next launch
        }
        __syncthreads();
        // Epilogue: the Cartesian block to shared memory, bra (and, Cartesian,
        // ket) output transform, stores.
#pragma unroll
        for (int k = 0; k < kGenAcc; k++) {
            const int e = tid + kGenThreads * k;
            if (e < n_ent) {
                const int rk = e / g.ko_chunk;
                sBase[sIJ[rk] * g.ko_chunk + (e - rk * g.ko_chunk)] = acc[k];
            }
        }
        __syncthreads();
        const size_t obase = (size_t)__ldg(map.out_begin + m);
        double wsum = 0.0;  // this thread's stored values (optional per-molecule checksum)
        const int nj_c = ncart(g.lj);
        for (int e = tid; e < nkoc * g.n_io * g.n_jo; e += kGenThreads) {
            const int kl = e / (g.n_io * g.n_jo), IJ = e - kl * (g.n_io * g.n_jo);
            const int I = IJ / g.n_jo, J = IJ - I * g.n_jo;
            const int ko = ko0 + kl;
            const double knorm = (g.spherical || g.point) ? 1.0 : c_cart_norm[c_cart_norm_offset[g.lk] + ko];
            double v = 0.0;
            for (int ca = 0; ca < ncart(g.li); ca++) {
                const double wi = g.spherical ? c_sph_coef[c_sph_offset[g.li] + I * ncart(g.li) + ca]
                                              : (I == ca ? c_cart_norm[c_cart_norm_offset[g.li] + ca] : 0.0);
                if (wi == 0.0) continue;
                double vj = 0.0;
                for (int cb = 0; cb < nj_c; cb++) {
                    const double wj = g.spherical ? c_sph_coef[c_sph_offset[g.lj] + J * nj_c + cb]
                                                  : (J == cb ? c_cart_norm[c_cart_norm_offset[g.lj] + cb] : 0.0);
                    if (wj != 0.0) vj = fma(wj, sBase[(ca * nj_c + cb) * g.ko_chunk + kl], vj);
                }
                v = fma(wi, vj, v);
            }
            const size_t row = (((size_t)sp_k * g.n_io + I) * g.n_jo + J) * g.n_ko + ko;
            out[obase + row * n_aux + a_local] = v * knorm;
            wsum += v * knorm;
        }
        if (map.checksum && wsum != 0.0) atomicAdd(map.checksum + m, wsum);
    }
}

int general_max_classes() { return kGenMaxClasses; }

int general_chunks(int li, int lj, int lk, bool point, bool spherical) {
    return general_shape(li, lj, lk, point, spherical).n_chunks;
}

// E tables of a pair class for the general kernel: one thread per (primitive
// pair, axis), 3 (x, y, z) x (l_i+1)(l_j+1)(l_i+l_j+1) doubles per primitive pair.
__global__ void general_e_table_kernel(int li, int lj, BraTable bra, int n_prim, double* __restrict__ out) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= 3 * n_prim) return;
    const int pp = w / 3, d = w - 3 * pp;
    // the primitive pair's shell pair: last g with grp_begin[g] <= pp
    int lo = 0, hi = bra.n_group - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(bra.grp_begin + mid) <= pp) lo = mid;
        else hi = mid - 1;
    }
    const int nea = (li + 1) * (lj + 1) * (li + lj + 1);
    const double4 AB = bra.grp_AB[lo];
    const double4 PA = bra.prim_PA[pp];
    const double pa_d = d == 0 ? PA.x : (d == 1 ? PA.y : PA.z);
    const double ab_d = d == 0 ? AB.x : (d == 1 ? AB.y : AB.z);
    general_e_axis(li, lj, pa_d, ab_d, 0.5 / bra.prim_P[pp].w, out + ((size_t)pp * 3 + d) * nea);
}

int general_e_doubles(int li, int lj) { return 3 * (li + 1) * (lj + 1) * (li + lj + 1); }

int launch_general_e_table(int li, int lj, const BraTable& bra, int n_prim, double* out, cudaStream_t s) {
    if (li < 0 || li > lj || li + lj > 2 * kMaxOrbitalL) return 1;
    if (bra.n_group == 0 || n_prim <= 0) return 0;
    if (n_prim > 0x7fffffff / 3) return 3;
    general_e_table_kernel<<<(3 * n_prim + 127) / 128, 128, 0, s>>>(li, lj, bra, n_prim, out);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int general_block_entries(int li, int lj, int lk, bool point, bool spherical) {
    const GenShape g = general_shape(li, lj, lk, point, spherical);
    return g.nij * g.ko_chunk;
}

double general_item_cost(int li, int lj, int lk, bool point, bool spherical) {
    const GenShape g = general_shape(li, lj, lk, point, spherical);
    // per unit: tetrahedron, ket and bra work of one chunk of ket components
    return (double)(g.nr + g.nhb * g.ko_chunk * g.nkc / 2 + g.nij * g.ko_chunk * g.nhb / 4 + 4 * (g.L + 1));
}

static bool general_class_ok(int li, int lj, int lk, bool point) {
    return li >= 0 && li <= lj && lj <= kMaxAuxL && li + lj <= 2 * kMaxOrbitalL && lk >= 0 && lk <= kMaxAuxL &&
           li + lj + (point ? 0 : lk) <= kGenMaxL;
}

int launch_general_multi(const GenClassSpec* specs, int n, bool spherical, const int2* perm, double omega,
                         double* out, int* counter, cudaStream_t s) {
    if (n <= 0) return 0;
    if (n > kGenMaxClasses) return 3;
    GenLaunch lp{};
    lp.n_classes = n;
    size_t smem = 0;
    long long total = 0;
    for (int c = 0; c < n; c++) {
        const GenClassSpec& sp = specs[c];
        if (!general_class_ok(sp.li, sp.lj, sp.lk, sp.point)) return 1;
        GenClassDesc& d = lp.cls[c];
        d.g = general_shape(sp.li, sp.lj, sp.lk, sp.point, spherical);
        d.bra = sp.bra;
        d.ket = sp.ket;
        d.map = sp.map;
        d.status = sp.status;
        if (sp.n_splits < 1 || sp.n_splits > kGenMaxSplits || (sp.n_splits > 1 && (!sp.partial || !sp.arrive)))
            return 3;
        d.g.n_splits = sp.n_splits;
        d.partial = sp.partial;
        d.etab = sp.etab;
        d.arrive = sp.arrive;
        lp.item0[c] = (int)total;
        total += sp.n_items;
        smem = std::max(smem, sizeof(double) * (size_t)d.g.smem_dbl);
    }
    lp.item0[n] = (int)total;
    if (total > 0x7fffffffLL) return 3;
    if (total == 0) return 0;
    if (smem > kGenMaxSmem) return 3;
    const double* table = boys_table_device();
    if (!table) return 2;
    // the shared-memory limit is raised once per device to the most any class takes
    static std::atomic<int> configured[kMaxDevices];
    if (persistent_grid(reinterpret_cast<const void*>(general_kernel), kGenThreads, kGenMaxSmem, configured) <= 0)
        return 2;
    int per_sm = 0, sms = 0;
    const int dev = current_device();
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, general_kernel, kGenThreads, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 2;
    const int grid = (int)std::min<long long>(total, (long long)std::max(1, per_sm) * sms);
    general_kernel<<<grid, kGenThreads, smem, s>>>(table, lp, perm, omega, out, counter, (int)total);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int launch_general(int li, int lj, int lk, bool point, bool spherical, const BraTable& bra, const KetTable& ket,
                   const BatchMap& map, int total_items, double omega, double* out, int* counter, cudaStream_t s) {
    if (!general_class_ok(li, lj, lk, point)) return 1;
    GenClassSpec sp{li, lj, point ? 0 : lk, point, bra, ket, map, total_items, counter + 1};
    return launch_general_multi(&sp, 1, spherical, nullptr, omega, out, counter, s);
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
