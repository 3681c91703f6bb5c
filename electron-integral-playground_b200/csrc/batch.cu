// Batched (mu nu|P) over many molecules: the eip_batch_* C ABI.
//
// A batch holds the pair and auxiliary tables of many molecules (the same
// structure-of-arrays format the reference ABI takes, one call per molecule
// and class), builds device-resident tables once (primitive pairs grouped by
// contracted shell pair, auxiliary primitives by shell, all molecules of one
// class concatenated), and captures ONE CUDA graph per batch that runs:
//   zero the work counters and checksums -> E-table kernels of every pair
//   class -> every (l_i, l_j | l_k) class kernel over all molecules at once
//   (persistent, atomic work list), forked over several streams so classes
//   overlap.
// Classes outside the fast kernels' range run the general kernel
// (k_generic.cu) over the same kind of multi-molecule work list, inside the
// same graph.
// Point charges (eip_batch_add_charges) form one more ket class, key
// kPointKet: the nuclear-attraction integrals V[mu nu C] of unit charges, run
// by the same kernels with a point-charge ket (l_k = 0, one block per charge).
// Output: one packed block per (molecule, class), offsets from
// eip_batch_block(); see k3c_fast.cuh for the layout.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <parallel/algorithm>
#include <map>
#include <numeric>
#include <vector>

#include "eip_common.cuh"
#include "eip_internal.h"
#include "../../include/eip_b200.h"

namespace eip {
namespace {

struct PairIn {
    std::vector<double> P, A, B, coef;
    std::vector<int> ia, ja;
};
struct AuxIn {
    std::vector<double> C, coef;
    std::vector<int> start;
};

// Ket-class key of point charges in the per-molecule auxiliary maps.
constexpr int kPointKet = EIP_POINT_CHARGES;

struct ClassPlan {
    int li, lj, lk;     // lk = kPointKet for point charges
    bool point = false;
    bool fast;
    int gen_chunks = 1;  // general kernel (not fast): items per block (ket-component chunks x splits)
    int gen_splits = 1;  // general kernel: items per (block, chunk), each over a share of the units
    size_t split_off = 0, arrive_off = 0;  // split classes: partial blocks and arrival counters
    int total_items = 0;
    BraTable bra{};
    KetTable ket{};
    BatchMap map{};
    int* counter = nullptr;
    // mixed precision: FP32 work list (shell pairs under the bound threshold)
    int total_items32 = 0;
    BatchMap map32{};
    int* counter32 = nullptr;
    long long triplets32 = 0, triplets64 = 0;
    int n_sp_total32 = 0;
    std::vector<int> n64, n32;          // per molecule: shell pairs on the FP64 / FP32 list
    // auxiliary window (eip_batch_window_plan): per molecule output offset and shells
    size_t win_off = 0;                 // this plan's arrays in the window buffers
    int win_items64 = 0, win_items32 = 0;
    std::vector<long long> win_out;
    std::vector<int> win_start, win_count;
    std::vector<long long> out_begin;   // per molecule
    std::vector<int> n_sp, n_auxsh;     // per molecule
    std::vector<int> sp0, aux0;         // per molecule (global indices in class tables)
    long long out_elems = 0;
    double flops_weight = 0;            // for scheduling order
};

template <typename T>
T* at(void* base, size_t off) {
    return reinterpret_cast<T*>(static_cast<char*>(base) + off);
}

struct Layout {
    size_t total = 0;
    size_t add(size_t bytes) {
        size_t off = total;
        total += (bytes + 255) & ~size_t(255);
        return off;
    }
};

}  // namespace
}  // namespace eip

using namespace eip;

struct eip_batch {
    int n_mol = 0;
    int device = -1;       // device the batch was built on; its calls run there
    bool spherical = true;
    double omega = 0.0;
    int precision = 0;     // 0 FP64, 1 mixed (FP32 for bounded shell pairs)
    // streams the class kernels are forked over: one by default, since two
    // persistent class kernels sharing the GPU slow each other down (the
    // 64-molecule step measured 290 ms on one stream, 304 ms on four)
    int n_streams = 1;
    double fp32_tau = 0.0;
    std::vector<std::map<std::pair<int, int>, PairIn>> pairs;  // per molecule
    std::vector<std::map<int, AuxIn>> aux;                     // per molecule
    bool built = false;
    cudaStream_t stream = nullptr;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> events;
    void* h_tables = nullptr;  // pinned copy of every device table (uploaded by eip_batch_upload)
    void* d_tables = nullptr;
    size_t table_bytes = 0;
    size_t device_bytes = 0;  // device memory of the tables, E tables, window maps and work lists
    double* d_etab = nullptr;
    double* d_out = nullptr;
    bool own_out = false;
    double* d_checksum = nullptr;
    long long out_elems = 0;
    std::vector<ClassPlan> plans;
    std::map<std::pair<int, int>, BraTable> bra_by_class;
    std::map<std::pair<int, int>, size_t> etab_offset;
    std::map<std::pair<int, int>, std::vector<int>> bra_sp_begin;  // per molecule prefix
    std::map<int, std::vector<int>> ket_aux_begin;
    std::map<int, std::vector<int>> ket_start;  // per class: first function of every auxiliary shell
    // auxiliary-window runs: per-plan maps in a ring of kWinSlots pinned buffers
    // mirrored on the device, so a window can be planned while earlier ones run
    static constexpr int kWinSlots = 4;
    void* h_win = nullptr;
    void* d_win = nullptr;
    size_t win_bytes = 0;  // one slot
    int win_slot = 0;      // slot of the planned window
    int win_next = 0;
    cudaEvent_t win_uploaded[kWinSlots] = {};  // the slot's last upload has been read
    bool win_pending[kWinSlots] = {};
    bool win_planned = false;
    bool win_charges = false;
    long long win_elems = 0;
    bool etab_ready = false;
    // general (non-fast) classes: launched together, up to
    // general_max_classes() per launch; per group its plan indices and the device work counter, and
    // (when not too many items) a heaviest-first order of its items
    std::vector<std::vector<int>> gen_groups;
    int* d_gen = nullptr;              // [group][4] counters, then the orders
    double* d_split = nullptr;         // partial blocks of the split general classes
    double* d_gen_etab = nullptr;      // E tables of the pair classes that general classes use
    std::map<std::pair<int, int>, size_t> gen_etab_offset;
    std::map<std::pair<int, int>, int> gen_etab_nprim;  // primitive pairs of those pair classes
    int* d_arrive = nullptr;           // their arrival counters (0 between launches)
    std::vector<size_t> gen_perm_off;  // per group, int2 offset into the orders (or SIZE_MAX)
    // density-fitting plan (eip_batch_df_plan): block list on the device
    DfBlock* d_df = nullptr;
    DfGather* d_dfg = nullptr;  // the gathered c vectors of the J contraction
    double* d_cg = nullptr;
    int df_blocks = 0, df_items = 0, df_gathers = 0;
    long long df_gather_elems = 0;
    long long df_ao2 = 0, df_aux = 0;  // total n_ao^2 and n_aux over the molecules
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long launches_per_run = 0;
    char err[256] = "";
};

namespace {

// Makes the batch's device current for one call and restores the caller's.
struct OnDevice {
    int saved = -1;
    bool switched = false;
    bool ok = true;
    explicit OnDevice(const eip_batch* b) {
        if (!b || b->device < 0 || cudaGetDevice(&saved) != cudaSuccess || saved == b->device) return;
        ok = cudaSetDevice(b->device) == cudaSuccess;
        switched = ok;
    }
    ~OnDevice() {
        if (switched) cudaSetDevice(saved);
    }
};

int fail(eip_batch* b, const char* what, cudaError_t e) {
    snprintf(b->err, sizeof b->err, "%s: %s", what, e == cudaSuccess ? "invalid" : cudaGetErrorString(e));
    fprintf(stderr, "[eip batch] %s\n", b->err);
    return 2;
}

void group_indices(const int* ia, const int* ja, int n, std::vector<int>& order, std::vector<int>& begin,
                   std::vector<int>& gi, std::vector<int>& gj) {
    order.resize(n);
    std::iota(order.begin(), order.end(), 0);
    auto less = [&](int x, int y) {
        const int jx = ja ? ja[x] : 0, jy = ja ? ja[y] : 0;
        return ia[x] != ia[y] ? ia[x] < ia[y] : jx < jy;
    };
    // large tables (a big molecule's pairs): the multi-threaded stable sort
    if (n > (1 << 16)) __gnu_parallel::stable_sort(order.begin(), order.end(), less);
    else std::stable_sort(order.begin(), order.end(), less);
    begin.clear();
    gi.clear();
    gj.clear();
    for (int k = 0; k < n; k++) {
        const int p = order[k];
        const int jp = ja ? ja[p] : 0;
        if (k == 0 || ia[p] != gi.back() || jp != gj.back()) {
            begin.push_back(k);
            gi.push_back(ia[p]);
            gj.push_back(jp);
        }
    }
    begin.push_back(n);
}

// Upper bound of |(ab|ab)|^(1/2) and of the overlap of one primitive pair, the
// construction of the reference front end (pair_utility.py:38-66) with the
// distance shift applied once: 2 |c_a c_b| (la/2ea)^(la/2) (lb/2eb)^(lb/2)
// exp(-ab/p d^2) max((pi/p)^1.5, 2^0.25 (pi/p)^1.25), d = max(|AB| - sqrt(la/2a)
// - sqrt(lb/2b), 0); |c_a c_b| recovered from c_ab = c_a c_b exp(-ab/p |AB|^2).
double pair_bound(const double* A, const double* B, double coef, int la, int lb) {
    // A one-centre "pair" (an s function of exponent 0 times one Gaussian: the
    // bra of the two-centre metric (P|Q) run as a three-centre class) gets an
    // infinite bound: the metric, which feeds a Cholesky factorisation, stays
    // FP64 in mixed mode.
    if (A[3] == 0.0 && la == 0) return HUGE_VAL;
    const double a = A[3], b = B[3], p = a + b, mu = a * b / p;
    const double dx = A[0] - B[0], dy = A[1] - B[1], dz = A[2] - B[2];
    const double ab2 = dx * dx + dy * dy + dz * dz, ab = sqrt(ab2);
    double d = ab - sqrt(la / (2.0 * a)) - sqrt(lb / (2.0 * b));
    if (d < 0.0) d = 0.0;
    double f = 2.0 * fabs(coef) * exp(mu * (ab2 - d * d));
    if (la > 0) f *= pow(la / (2.0 * M_E * a), la / 2.0);
    if (lb > 0) f *= pow(lb / (2.0 * M_E * b), lb / 2.0);
    return f * fmax(pow(M_PI / p, 1.5), pow(2.0, 0.25) * pow(M_PI / p, 1.25));
}

// Same construction for one auxiliary primitive: |c| 2 (l/2eq)^(l/2) (2 pi^(5/2) / (q^2 sqrt(2q)))^(1/2).
double aux_bound(double q, double coef, int l) {
    double f = 2.0 * fabs(coef) * sqrt(2.0 * pow(M_PI, 2.5) / (q * q * sqrt(2.0 * q)));
    if (l > 0) f *= pow(l / (2.0 * M_E * q), l / 2.0);
    return f;
}

// Largest sum of |coefficients| of a row of the output transform of one l.
double transform_gain(int l, bool spherical) {
    double g = 1.0;
    for (int m = 0; m < (spherical ? nsph(l) : ncart(l)); m++) {
        double r = 0.0;
        for (int c = 0; c < ncart(l); c++)
            r += spherical ? fabs(eip_sph_coef[eip_sph_offset[l] + m * ncart(l) + c])
                           : (m == c ? eip_cart_norm[eip_cart_norm_offset[l] + c] : 0.0);
        g = fmax(g, r);
    }
    return g;
}

}  // namespace

extern "C" {

int eip_batch_set_streams(eip_batch* b, int n_streams) {
    if (!b || b->exec || !b->side.empty() || n_streams < 1 || n_streams > 8) return 2;
    b->n_streams = n_streams;
    return 0;
}

int eip_batch_set_precision(eip_batch* b, int mode, double fp32_threshold) {
    if (!b || b->built || mode < 0 || mode > 1 || !(fp32_threshold >= 0.0)) return 2;
    b->precision = mode;
    b->fp32_tau = fp32_threshold;
    return 0;
}

eip_batch* eip_batch_create(int n_molecules, bool spherical, double omega) {
    if (n_molecules <= 0 || omega < 0.0) return nullptr;
    eip_batch* b = new eip_batch;
    b->n_mol = n_molecules;
    b->spherical = spherical;
    b->omega = omega;
    b->pairs.resize(n_molecules);
    b->aux.resize(n_molecules);
    return b;
}

const char* eip_batch_error(eip_batch* b) { return b ? b->err : "null batch"; }

int eip_batch_add_pairs(eip_batch* b, int mol, int i_L, int j_L, const double* P_p, const double* A_a,
                        const double* B_b, const double* coefficient, const int* i_ao_start, const int* j_ao_start,
                        int n_pair) {
    if (!b || b->built || mol < 0 || mol >= b->n_mol || n_pair < 0) return 2;
    if (i_L < 0 || i_L > j_L || j_L > kMaxOrbitalL) return 1;
    PairIn& p = b->pairs[mol][{i_L, j_L}];
    p.P.insert(p.P.end(), P_p, P_p + 4 * (size_t)n_pair);
    p.A.insert(p.A.end(), A_a, A_a + 4 * (size_t)n_pair);
    p.B.insert(p.B.end(), B_b, B_b + 4 * (size_t)n_pair);
    p.coef.insert(p.coef.end(), coefficient, coefficient + n_pair);
    p.ia.insert(p.ia.end(), i_ao_start, i_ao_start + n_pair);
    p.ja.insert(p.ja.end(), j_ao_start, j_ao_start + n_pair);
    return 0;
}

int eip_batch_add_aux(eip_batch* b, int mol, int k_L, const double* A_a, const double* coefficient,
                      const int* aux_start, int n_primitive) {
    if (!b || b->built || mol < 0 || mol >= b->n_mol || n_primitive < 0) return 2;
    if (k_L < 0 || k_L > kMaxAuxL) return 1;
    AuxIn& a = b->aux[mol][k_L];
    a.C.insert(a.C.end(), A_a, A_a + 4 * (size_t)n_primitive);
    a.coef.insert(a.coef.end(), coefficient, coefficient + n_primitive);
    a.start.insert(a.start.end(), aux_start, aux_start + n_primitive);
    return 0;
}

int eip_batch_add_charges(eip_batch* b, int mol, const double* position, int n_charge) {
    if (!b || b->built || mol < 0 || mol >= b->n_mol || n_charge < 0) return 2;
    AuxIn& a = b->aux[mol][kPointKet];
    const int first = (int)a.start.size();
    for (int c = 0; c < n_charge; c++) {
        a.C.insert(a.C.end(), {position[3 * (size_t)c], position[3 * (size_t)c + 1], position[3 * (size_t)c + 2], 1.0});
        a.coef.push_back(1.0);
        a.start.push_back(first + c);
    }
    return 0;
}

int eip_batch_build(eip_batch* b) {
    if (!b || b->built) return 2;
    if (int rc = eip_init(-1)) return fail(b, eip_last_error(), cudaSuccess) ? rc : rc;
    b->device = current_device();
    if (b->device < 0) return fail(b, "no usable CUDA device", cudaErrorInvalidDevice);
    if (int rc = ensure_device_tables()) return fail(b, "constant tables", (cudaError_t)rc);
    cudaError_t e;
    // ---- which classes exist
    std::map<std::pair<int, int>, int> pair_classes;
    std::map<int, int> aux_classes;
    for (int m = 0; m < b->n_mol; m++) {
        for (auto& kv : b->pairs[m]) pair_classes[kv.first] = 1;
        for (auto& kv : b->aux[m]) aux_classes[kv.first] = 1;
    }
    // ---- group and lay out every table
    struct BraHost {
        std::vector<int> begin;
        std::vector<int2> ao;
        std::vector<double4> AB, P, PA;
        std::vector<int> sp_begin;  // per molecule prefix (n_mol + 1)
        std::vector<double> bound;  // per shell pair: sum of primitive pair bounds
    };
    struct KetHost {
        std::vector<int> begin, start;
        std::vector<double4> C;
        std::vector<double> coef;
        std::vector<int> aux_begin;
        std::vector<double> max_bound;  // per molecule: largest auxiliary shell bound
    };
    std::map<std::pair<int, int>, BraHost> bh;
    std::map<int, KetHost> kh;
    std::vector<int> order, gb, gi, gj;
    for (auto& pc : pair_classes) {
        BraHost& H = bh[pc.first];
        H.begin.push_back(0);
        H.sp_begin.push_back(0);
        for (int m = 0; m < b->n_mol; m++) {
            auto it = b->pairs[m].find(pc.first);
            if (it != b->pairs[m].end() && !it->second.ia.empty()) {
                const PairIn& p = it->second;
                const int n = (int)p.ia.size();
                group_indices(p.ia.data(), p.ja.data(), n, order, gb, gi, gj);
                const int prim0 = (int)H.P.size();
                const int ng = (int)gb.size() - 1;
                const size_t g0 = H.ao.size();
                H.ao.resize(g0 + ng);
                H.AB.resize(g0 + ng);
                H.bound.resize(g0 + ng);
                H.begin.resize(g0 + 1 + ng);
                H.P.resize((size_t)prim0 + n);
                H.PA.resize((size_t)prim0 + n);
                const int li = pc.first.first, lj = pc.first.second;
                // each group and each primitive is independent: fill in parallel
#pragma omp parallel for schedule(dynamic, 256)
                for (int g = 0; g < ng; g++) {
                    H.ao[g0 + g] = make_int2(gi[g], gj[g]);
                    const int q = order[gb[g]];
                    H.AB[g0 + g] = make_double4(p.A[4 * q] - p.B[4 * q], p.A[4 * q + 1] - p.B[4 * q + 1],
                                                p.A[4 * q + 2] - p.B[4 * q + 2], 0.0);
                    H.begin[g0 + 1 + g] = prim0 + gb[g + 1];
                    double qb = 0.0;
                    for (int k = gb[g]; k < gb[g + 1]; k++) {
                        const int r = order[k];
                        qb += pair_bound(&p.A[4 * r], &p.B[4 * r], p.coef[r], li, lj);
                    }
                    H.bound[g0 + g] = qb;
                }
#pragma omp parallel for schedule(static)
                for (int k = 0; k < n; k++) {
                    const int q = order[k];
                    const double* P = &p.P[4 * q];
                    const double* A = &p.A[4 * q];
                    H.P[(size_t)prim0 + k] = make_double4(P[0], P[1], P[2], P[3]);
                    H.PA[(size_t)prim0 + k] = make_double4(P[0] - A[0], P[1] - A[1], P[2] - A[2], p.coef[q]);
                }
            }
            H.sp_begin.push_back((int)H.ao.size());
        }
    }
    for (auto& ac : aux_classes) {
        KetHost& H = kh[ac.first];
        H.begin.push_back(0);
        H.aux_begin.push_back(0);
        for (int m = 0; m < b->n_mol; m++) {
            double qmax = 0.0;
            auto it = b->aux[m].find(ac.first);
            if (it != b->aux[m].end() && !it->second.start.empty()) {
                const AuxIn& a = it->second;
                const int n = (int)a.start.size();
                group_indices(a.start.data(), nullptr, n, order, gb, gi, gj);
                const int prim0 = (int)H.C.size();
                for (size_t g = 0; g + 1 < gb.size(); g++) {
                    H.start.push_back(gi[g]);
                    H.begin.push_back(prim0 + gb[g + 1]);
                    double qa = 0.0;
                    for (int k = gb[g]; k < gb[g + 1]; k++)
                        if (ac.first != kPointKet) qa += aux_bound(a.C[4 * order[k] + 3], a.coef[order[k]], ac.first);
                    qmax = fmax(qmax, qa);
                }
                for (int k = 0; k < n; k++) {
                    const int q = order[k];
                    H.C.push_back(make_double4(a.C[4 * q], a.C[4 * q + 1], a.C[4 * q + 2], a.C[4 * q + 3]));
                    H.coef.push_back(a.coef[q]);
                }
            }
            H.max_bound.push_back(qmax);
            H.aux_begin.push_back((int)H.start.size());
        }
    }
    // ---- plans (one per pair class x aux class)
    for (auto& pc : pair_classes)
        for (auto& ac : aux_classes) {
            ClassPlan pl;
            pl.li = pc.first.first;
            pl.lj = pc.first.second;
            pl.lk = ac.first;
            pl.point = ac.first == kPointKet;
            const int lk = pl.point ? 0 : pl.lk;
            const BraHost& B = bh[pc.first];
            const KetHost& K = kh[ac.first];
            // The fast kernels give each lane one auxiliary shell of a tile of
            // 32: when the molecules hold so few shells of the class that most
            // lanes would idle (below a quarter in use), the class runs on the
            // general kernel, which spreads one block over a whole CTA.
            long long used = 0, slots = 0;
            for (int m = 0; m < b->n_mol; m++) {
                const long long nsp = B.sp_begin[m + 1] - B.sp_begin[m], nax = K.aux_begin[m + 1] - K.aux_begin[m];
                used += nsp * nax;
                slots += nsp * ((nax + 31) / 32) * 32;
            }
            pl.fast = b->spherical && fast3c_supported(pl.li, pl.lj, lk) && 4 * used >= slots;
            if (!pl.fast) {
                // A general item is one CTA over every unit (primitive pair x
                // auxiliary primitive) of its block; when a class's blocks hold
                // many units (high-l shells of 1-8 primitives), its few heavy
                // items would run long after the rest of the launch, so each
                // block is split into items of about kUnitsPerSplit units.
                const int kch = general_chunks(pl.li, pl.lj, lk, pl.point, b->spherical);
                long long max_units = 0, base_items = 0;
                for (int m = 0; m < b->n_mol; m++) {
                    int max_pp = 0, max_kp = 0;
                    for (int sp = B.sp_begin[m]; sp < B.sp_begin[m + 1]; sp++)
                        max_pp = std::max(max_pp, B.begin[sp + 1] - B.begin[sp]);
                    for (int a = K.aux_begin[m]; a < K.aux_begin[m + 1]; a++)
                        max_kp = std::max(max_kp, K.begin[a + 1] - K.begin[a]);
                    max_units = std::max(max_units, (long long)max_pp * max_kp);
                    base_items += (long long)(B.sp_begin[m + 1] - B.sp_begin[m]) *
                                  (K.aux_begin[m + 1] - K.aux_begin[m]) * kch;
                }
                constexpr int kSplitMinUnits = 64, kUnitsPerSplit = 32, kMaxSplits = 16;
                constexpr long long kSplitScratchMax = 64LL << 20;  // doubles of partial blocks per class
                int S = max_units >= kSplitMinUnits
                            ? (int)std::min<long long>(kMaxSplits, (max_units + kUnitsPerSplit - 1) / kUnitsPerSplit)
                            : 1;
                const long long ent = general_block_entries(pl.li, pl.lj, lk, pl.point, b->spherical);
                while (S > 1 && base_items * S * ent > kSplitScratchMax) S /= 2;
                pl.gen_splits = S;
                pl.gen_chunks = kch * S;
            }
            const int ni = b->spherical ? nsph(pl.li) : ncart(pl.li), nj = b->spherical ? nsph(pl.lj) : ncart(pl.lj),
                      nk = b->spherical ? nsph(lk) : ncart(lk);
            long long items = 0;
            for (int m = 0; m < b->n_mol; m++) {
                const int nsp = B.sp_begin[m + 1] - B.sp_begin[m], nax = K.aux_begin[m + 1] - K.aux_begin[m];
                pl.n_sp.push_back(nsp);
                pl.n_auxsh.push_back(nax);
                pl.sp0.push_back(B.sp_begin[m]);
                pl.aux0.push_back(K.aux_begin[m]);
                pl.out_begin.push_back(b->out_elems);
                const long long blk = (long long)nsp * ni * nj * nk * nax;
                b->out_elems += blk;
                pl.out_elems += blk;
                items += pl.fast ? (long long)nsp * ((nax + 31) / 32) : (long long)nsp * nax * pl.gen_chunks;
            }
            if (items > 0x7fffffffLL) return fail(b, "too many work items in one class", cudaSuccess);
            pl.total_items = (int)items;
            pl.flops_weight = (double)pl.out_elems * (pl.li + pl.lj + lk + 1);
            b->plans.push_back(pl);
        }
    // ---- one pinned buffer with every table, mirrored on the device
    Layout L;
    struct BraOff { size_t beg, ao, ab, p, pa, spb; };
    struct KetOff { size_t beg, st, c, co, axb; };
    std::map<std::pair<int, int>, BraOff> bo;
    std::map<int, KetOff> ko;
    for (auto& kv : bh) {
        const BraHost& H = kv.second;
        bo[kv.first] = BraOff{L.add(sizeof(int) * H.begin.size()), L.add(sizeof(int2) * H.ao.size()),
                              L.add(sizeof(double4) * H.AB.size()), L.add(sizeof(double4) * H.P.size()),
                              L.add(sizeof(double4) * H.PA.size()), L.add(sizeof(int) * H.sp_begin.size())};
    }
    for (auto& kv : kh) {
        const KetHost& H = kv.second;
        ko[kv.first] = KetOff{L.add(sizeof(int) * H.begin.size()), L.add(sizeof(int) * H.start.size()),
                              L.add(sizeof(double4) * H.C.size()), L.add(sizeof(double) * H.coef.size()),
                              L.add(sizeof(int) * H.aux_begin.size())};
    }
    // Per-plan work maps: ints = [item_begin64 | list_begin64 | aux_begin | item_begin32 |
    // list_begin32 | sp_first] (n_mol + 1 each), 4 counters/status words, the
    // FP64 and FP32 shell-pair lists; then the 8-byte aligned out_begin array.
    const int nm = b->n_mol;
    std::vector<std::vector<int>> plan_ints(b->plans.size());
    std::vector<size_t> plan_off, plan_ob;
    for (size_t i = 0; i < b->plans.size(); i++) {
        ClassPlan& pl = b->plans[i];
        const BraHost& B = bh[{pl.li, pl.lj}];
        const KetHost& K = kh[pl.lk];
        const bool mixed = b->precision == 1 && pl.fast && !pl.point;
        const double gain = transform_gain(pl.li, b->spherical) * transform_gain(pl.lj, b->spherical) *
                            transform_gain(pl.point ? 0 : pl.lk, b->spherical);
        std::vector<int>& v = plan_ints[i];
        v.assign(6 * (nm + 1) + 4, 0);
        int* ib64 = &v[0];
        int* lb64 = &v[nm + 1];
        int* axb = &v[2 * (nm + 1)];
        int* ib32 = &v[3 * (nm + 1)];
        int* lb32 = &v[4 * (nm + 1)];
        int* spf = &v[5 * (nm + 1)];
        std::vector<int> list64, list32;
        for (int m = 0; m < nm; m++) {
            // work items per shell pair: tiles of 32 auxiliary shells (fast
            // kernels) or auxiliary shells x ket chunks (general kernel)
            const int tiles = pl.fast ? (pl.n_auxsh[m] + 31) / 32 : pl.n_auxsh[m] * pl.gen_chunks;
            int n64 = 0, n32 = 0;
            for (int g = B.sp_begin[m]; g < B.sp_begin[m + 1]; g++) {
                const bool f32 = mixed && B.bound[g] * K.max_bound[m] * gain < b->fp32_tau;
                (f32 ? list32 : list64).push_back(g);
                (f32 ? n32 : n64)++;
            }
            pl.triplets32 += (long long)n32 * pl.n_auxsh[m];
            pl.triplets64 += (long long)n64 * pl.n_auxsh[m];
            pl.n64.push_back(n64);
            pl.n32.push_back(n32);
            ib64[m + 1] = ib64[m] + n64 * tiles;
            ib32[m + 1] = ib32[m] + n32 * tiles;
            lb64[m + 1] = lb64[m] + n64;
            lb32[m + 1] = lb32[m] + n32;
        }
        for (int m = 0; m <= nm; m++) {
            axb[m] = K.aux_begin[m];
            spf[m] = B.sp_begin[m];
        }
        if ((long long)ib64[nm] > 0x7fffffffLL || (long long)ib32[nm] > 0x7fffffffLL)
            return fail(b, "too many work items in one class", cudaSuccess);
        pl.total_items = ib64[nm];
        pl.total_items32 = ib32[nm];
        pl.n_sp_total32 = (int)list32.size();
        v.insert(v.end(), list64.begin(), list64.end());
        v.insert(v.end(), list32.begin(), list32.end());
        const size_t ints_bytes = (sizeof(int) * v.size() + 7) & ~size_t(7);
        plan_off.push_back(L.add(ints_bytes + sizeof(long long) * nm));
        plan_ob.push_back(plan_off.back() + ints_bytes);
    }
    size_t etab_total = 0;
    for (auto& kv : bh) {
        b->etab_offset[kv.first] = etab_total;
        etab_total += e_table_doubles(kv.first.first, kv.first.second) * kv.second.P.size();
    }
    b->table_bytes = L.total;
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(b, "stream", e);
    if ((e = cudaMallocHost(&b->h_tables, L.total)) != cudaSuccess) return fail(b, "pinned tables", e);
    if ((e = cudaMalloc(&b->d_tables, L.total)) != cudaSuccess) return fail(b, "device tables", e);
    if ((e = cudaMalloc((void**)&b->d_etab, sizeof(double) * std::max<size_t>(etab_total, 1))) != cudaSuccess)
        return fail(b, "E tables", e);
    if ((e = cudaMalloc((void**)&b->d_checksum, sizeof(double) * b->n_mol)) != cudaSuccess)
        return fail(b, "checksums", e);
    b->device_bytes += L.total + sizeof(double) * (std::max<size_t>(etab_total, 1) + b->n_mol);
    void* h = b->h_tables;
    void* d = b->d_tables;
    for (auto& kv : bh) {
        const BraHost& H = kv.second;
        const BraOff& o = bo[kv.first];
        memcpy(at<int>(h, o.beg), H.begin.data(), sizeof(int) * H.begin.size());
        memcpy(at<int2>(h, o.ao), H.ao.data(), sizeof(int2) * H.ao.size());
        memcpy(at<double4>(h, o.ab), H.AB.data(), sizeof(double4) * H.AB.size());
        memcpy(at<double4>(h, o.p), H.P.data(), sizeof(double4) * H.P.size());
        memcpy(at<double4>(h, o.pa), H.PA.data(), sizeof(double4) * H.PA.size());
        memcpy(at<int>(h, o.spb), H.sp_begin.data(), sizeof(int) * H.sp_begin.size());
        b->bra_by_class[kv.first] =
            BraTable{(int)H.ao.size(), at<int>(d, o.beg), at<int2>(d, o.ao), at<double4>(d, o.ab), at<double4>(d, o.p),
                     at<double4>(d, o.pa), b->d_etab + b->etab_offset[kv.first]};
        b->bra_sp_begin[kv.first] = H.sp_begin;
    }
    std::map<int, KetTable> ket_by_class;
    for (auto& kv : kh) {
        const KetHost& H = kv.second;
        const KetOff& o = ko[kv.first];
        memcpy(at<int>(h, o.beg), H.begin.data(), sizeof(int) * H.begin.size());
        memcpy(at<int>(h, o.st), H.start.data(), sizeof(int) * H.start.size());
        memcpy(at<double4>(h, o.c), H.C.data(), sizeof(double4) * H.C.size());
        memcpy(at<double>(h, o.co), H.coef.data(), sizeof(double) * H.coef.size());
        memcpy(at<int>(h, o.axb), H.aux_begin.data(), sizeof(int) * H.aux_begin.size());
        ket_by_class[kv.first] =
            KetTable{(int)H.start.size(), at<int>(d, o.beg), at<int>(d, o.st), at<double4>(d, o.c), at<double>(d, o.co)};
        b->ket_aux_begin[kv.first] = H.aux_begin;
        b->ket_start[kv.first] = H.start;
    }
    for (size_t i = 0; i < b->plans.size(); i++) {
        ClassPlan& pl = b->plans[i];
        const std::vector<int>& v = plan_ints[i];
        memcpy(at<int>(h, plan_off[i]), v.data(), sizeof(int) * v.size());
        memcpy(at<long long>(h, plan_ob[i]), pl.out_begin.data(), sizeof(long long) * nm);
        int* dp = at<int>(d, plan_off[i]);
        const long long* dob = at<long long>(d, plan_ob[i]);
        const bool mixed = b->precision == 1 && pl.fast && !pl.point;
        int* counters = dp + 6 * (nm + 1);
        const int* list64 = counters + 4;
        const int* list32 = list64 + (v.size() - 6 * (nm + 1) - 4) - pl.n_sp_total32;
        pl.bra = b->bra_by_class[{pl.li, pl.lj}];
        pl.ket = ket_by_class[pl.lk];
        pl.counter = counters;
        pl.counter32 = counters + 2;
        if (mixed) {
            pl.map = BatchMap{nm, dp, dp + (nm + 1), dp + 2 * (nm + 1), dob, nullptr, list64, dp + 5 * (nm + 1)};
            pl.map32 = BatchMap{nm, dp + 3 * (nm + 1), dp + 4 * (nm + 1), dp + 2 * (nm + 1), dob, nullptr, list32,
                                dp + 5 * (nm + 1)};
        } else {
            // all pairs in FP64: plain numbering, sp_begin = the molecule's first pair
            pl.map = BatchMap{nm, dp, dp + 5 * (nm + 1), dp + 2 * (nm + 1), dob, nullptr, nullptr, nullptr};
        }
    }
    // window maps: per plan [item_begin64 | item_begin32 (n_mol + 1 each) | aux start |
    // aux count (n_mol each)], then the 8-byte aligned out_begin (n_mol)
    {
        Layout W;
        for (ClassPlan& pl : b->plans) pl.win_off = W.add(sizeof(int) * (4 * nm + 2) + 8 + sizeof(long long) * nm);
        b->win_bytes = std::max<size_t>(W.total, 256);
        if ((e = cudaMallocHost(&b->h_win, b->win_bytes * eip_batch::kWinSlots)) != cudaSuccess)
            return fail(b, "pinned window maps", e);
        if ((e = cudaMalloc(&b->d_win, b->win_bytes * eip_batch::kWinSlots)) != cudaSuccess)
            return fail(b, "window maps", e);
        b->device_bytes += b->win_bytes * eip_batch::kWinSlots;
        for (int i = 0; i < eip_batch::kWinSlots; i++)
            if ((e = cudaEventCreateWithFlags(&b->win_uploaded[i], cudaEventDisableTiming)) != cudaSuccess)
                return fail(b, "event", e);
    }
    if ((e = cudaMemcpyAsync(d, h, L.total, cudaMemcpyHostToDevice, b->stream)) != cudaSuccess)
        return fail(b, "table upload", e);
    if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return fail(b, "table upload", e);
    // heaviest classes first in the graph
    std::sort(b->plans.begin(), b->plans.end(),
              [](const ClassPlan& x, const ClassPlan& y) { return x.flops_weight > y.flops_weight; });
    // general classes: groups of up to general_max_classes() per launch, each group's items in
    // order of decreasing work (primitive pairs x auxiliary primitives x the
    // class's work per unit), so that the launch does not end on a heavy item
    {
        std::vector<int> gen;
        for (size_t i = 0; i < b->plans.size(); i++)
            if (!b->plans[i].fast && b->plans[i].total_items > 0) gen.push_back((int)i);
        const size_t per = (size_t)general_max_classes();
        for (size_t k = 0; k < gen.size(); k += per)
            b->gen_groups.emplace_back(gen.begin() + k, gen.begin() + std::min(gen.size(), k + per));
        long long gen_items = 0;
        for (int i : gen) gen_items += b->plans[i].total_items;
        const bool order = gen_items > 0 && gen_items <= (8LL << 20);
        std::vector<int2> perm;
        for (const std::vector<int>& grp : b->gen_groups) {
            b->gen_perm_off.push_back(order ? perm.size() : SIZE_MAX);
            if (!order) continue;
            std::vector<std::pair<double, int2>> items;
            for (size_t c = 0; c < grp.size(); c++) {
                const ClassPlan& pl = b->plans[grp[c]];
                const BraHost& B = bh[{pl.li, pl.lj}];
                const KetHost& K = kh[pl.lk];
                const int lk = pl.point ? 0 : pl.lk;
                const double unit = general_item_cost(pl.li, pl.lj, lk, pl.point, b->spherical) / pl.gen_splits;
                int item = 0;
                for (int m = 0; m < b->n_mol; m++)
                    for (int sp = B.sp_begin[m]; sp < B.sp_begin[m + 1]; sp++)
                        for (int a = K.aux_begin[m]; a < K.aux_begin[m + 1]; a++)
                            for (int ch = 0; ch < pl.gen_chunks; ch++) {
                                const double w = (double)(B.begin[sp + 1] - B.begin[sp]) * (K.begin[a + 1] - K.begin[a]);
                                items.push_back({w * unit, make_int2((int)c, item++)});
                            }
            }
            std::stable_sort(items.begin(), items.end(),
                             [](const std::pair<double, int2>& x, const std::pair<double, int2>& y) {
                                 return x.first > y.first;
                             });
            for (auto& it : items) perm.push_back(it.second);
        }
        // E tables of the pair classes the general classes use (computed with
        // the fast classes' tables at every run)
        size_t gen_etab_doubles = 0;
        for (int i : gen) {
            const ClassPlan& pl = b->plans[i];
            const std::pair<int, int> pc{pl.li, pl.lj};
            if (b->gen_etab_offset.count(pc)) continue;
            b->gen_etab_offset[pc] = gen_etab_doubles;
            b->gen_etab_nprim[pc] = (int)bh[pc].P.size();
            gen_etab_doubles += (size_t)general_e_doubles(pl.li, pl.lj) * bh[pc].P.size();
        }
        if (gen_etab_doubles > 0) {
            if ((e = cudaMalloc((void**)&b->d_gen_etab, sizeof(double) * gen_etab_doubles)) != cudaSuccess)
                return fail(b, "general E tables", e);
            b->device_bytes += sizeof(double) * gen_etab_doubles;
        }
        // partial blocks and arrival counters of the split classes
        size_t split_doubles = 0, arrive_ints = 0;
        for (int i : gen) {
            ClassPlan& pl = b->plans[i];
            if (pl.gen_splits <= 1) continue;
            pl.split_off = split_doubles;
            pl.arrive_off = arrive_ints;
            split_doubles += (size_t)pl.total_items *
                             general_block_entries(pl.li, pl.lj, pl.point ? 0 : pl.lk, pl.point, b->spherical);
            arrive_ints += (size_t)pl.total_items / pl.gen_splits;
        }
        if (split_doubles > 0) {
            if ((e = cudaMalloc((void**)&b->d_split, sizeof(double) * split_doubles)) != cudaSuccess ||
                (e = cudaMalloc((void**)&b->d_arrive, sizeof(int) * arrive_ints)) != cudaSuccess ||
                (e = cudaMemset(b->d_arrive, 0, sizeof(int) * arrive_ints)) != cudaSuccess)
                return fail(b, "general split blocks", e);
            b->device_bytes += sizeof(double) * split_doubles + sizeof(int) * arrive_ints;
        }
        if (!b->gen_groups.empty()) {
            const size_t bytes = sizeof(int) * 4 * b->gen_groups.size() + sizeof(int2) * perm.size();
            if ((e = cudaMalloc((void**)&b->d_gen, bytes)) != cudaSuccess) return fail(b, "general work lists", e);
            b->device_bytes += bytes;
            if (!perm.empty() &&
                (e = cudaMemcpy(b->d_gen + 4 * b->gen_groups.size(), perm.data(), sizeof(int2) * perm.size(),
                                cudaMemcpyHostToDevice)) != cudaSuccess)
                return fail(b, "general work lists", e);
        }
    }
    b->built = true;
    return 0;
}

static size_t win_ob_off(int nm);

// The general-launch description of a plan over `map` (n_items items); for a
// split class also clears its arrival counters on stream s (they are left 0
// by every complete launch; the clear keeps an interrupted one from leaking
// into the next).
// The general kernel's E tables of every pair class a general class uses,
// on stream s (after the tables' upload, before the general launches).
static int launch_gen_etabs(eip_batch* b, cudaStream_t s, unsigned long long* launches = nullptr) {
    int rc = 0;
    for (const auto& kv : b->gen_etab_offset) {
        rc |= launch_general_e_table(kv.first.first, kv.first.second, b->bra_by_class[kv.first],
                                     b->gen_etab_nprim[kv.first], b->d_gen_etab + kv.second, s);
        if (launches) ++*launches;
    }
    return rc;
}

static GenClassSpec gen_spec(eip_batch* b, ClassPlan& pl, const BatchMap& map, int n_items, cudaStream_t s) {
    GenClassSpec sp{pl.li, pl.lj, pl.point ? 0 : pl.lk, pl.point, pl.bra, pl.ket, map, n_items, pl.counter + 1};
    auto et = b->gen_etab_offset.find({pl.li, pl.lj});
    if (et != b->gen_etab_offset.end()) sp.etab = b->d_gen_etab + et->second;
    if (pl.gen_splits > 1) {
        sp.n_splits = pl.gen_splits;
        sp.partial = b->d_split + pl.split_off;
        sp.arrive = b->d_arrive + pl.arrive_off;
        cudaMemsetAsync(sp.arrive, 0, sizeof(int) * (size_t)(pl.total_items / pl.gen_splits), s);
    }
    return sp;
}

// One multi-class launch per group of general classes (work maps: the plans'
// own, or the planned window's when win is set), on the side streams.
static int launch_general_groups(eip_batch* b, bool checksum, bool win, void* dw, double* out, int& launches) {
    int rc = 0;
    const int nm = b->n_mol;
    for (size_t g = 0; g < b->gen_groups.size(); g++) {
        std::vector<GenClassSpec> specs;
        cudaStream_t s = b->side[g % b->side.size()];
        for (int i : b->gen_groups[g]) {
            ClassPlan& pl = b->plans[i];
            cudaMemsetAsync(pl.counter, 0, 4 * sizeof(int), s);  // status word, on the launch's stream
            BatchMap map = pl.map;
            map.checksum = checksum ? b->d_checksum : nullptr;
            int n_items = pl.total_items;
            if (win) {
                const int* v = at<int>(dw, pl.win_off);
                map.item_begin = v;
                map.aux_begin = v + 2 * (nm + 1);
                map.aux_count = v + 2 * (nm + 1) + nm;
                map.out_begin = at<long long>(dw, pl.win_off + win_ob_off(nm));
                n_items = pl.win_items64;
            }
            specs.push_back(gen_spec(b, pl, map, n_items, s));
        }
        int* counter = b->d_gen + 4 * g;
        const int2* perm = (!win && b->gen_perm_off[g] != SIZE_MAX)
                               ? reinterpret_cast<const int2*>(b->d_gen + 4 * b->gen_groups.size()) + b->gen_perm_off[g]
                               : nullptr;
        cudaMemsetAsync(counter, 0, 4 * sizeof(int), s);
        rc |= launch_general_multi(specs.data(), (int)specs.size(), b->spherical, perm, b->omega, out, counter, s);
        launches++;
    }
    return rc;
}

long long eip_batch_output_elems(eip_batch* b) { return b && b->built ? b->out_elems : -1; }

int eip_batch_block(eip_batch* b, int mol, int i_L, int j_L, int k_L, long long* offset, int* n_pair_shells,
                    int* n_aux_shells) {
    if (!b || !b->built || mol < 0 || mol >= b->n_mol) return 2;
    for (const ClassPlan& pl : b->plans)
        if (pl.li == i_L && pl.lj == j_L && pl.lk == k_L) {
            *offset = pl.out_begin[mol];
            *n_pair_shells = pl.n_sp[mol];
            *n_aux_shells = pl.n_auxsh[mol];
            return 0;
        }
    return 1;
}

int eip_batch_bind_output(eip_batch* b, double* device_out) {
    if (!b || !b->built) return 2;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
    }
    if (b->own_out && b->d_out) cudaFree(b->d_out);
    b->own_out = false;
    b->d_out = device_out;
    return 0;
}

int eip_batch_alloc_output(eip_batch* b) {
    if (!b || !b->built) return 2;
    OnDevice on(b);
    if (!on.ok) return fail(b, "cudaSetDevice (batch device)", cudaErrorInvalidDevice);
    double* p = nullptr;
    cudaError_t e = cudaMalloc((void**)&p, sizeof(double) * std::max<long long>(b->out_elems, 1));
    if (e != cudaSuccess) return fail(b, "output allocation", e);
    eip_batch_bind_output(b, p);
    b->own_out = true;
    return 0;
}

double* eip_batch_output_device(eip_batch* b) { return b ? b->d_out : nullptr; }

static int capture(eip_batch* b, bool checksum) {
    cudaError_t e;
    const int n_side = b->n_streams;
    if (b->side.empty()) {
        for (int i = 0; i < n_side; i++) {
            cudaStream_t s;
            if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) return fail(b, "stream", e);
            b->side.push_back(s);
        }
        for (int i = 0; i < 2 * n_side + 1; i++) {
            cudaEvent_t ev;
            if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return fail(b, "event", e);
            b->events.push_back(ev);
        }
    }
    unsigned long long launches = 0;
    if ((e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return fail(b, "begin capture", e);
    int rc = 0;
    cudaMemsetAsync(b->d_checksum, 0, sizeof(double) * b->n_mol, b->stream);
    for (ClassPlan& pl : b->plans)
        cudaMemsetAsync(pl.counter, 0, 4 * sizeof(int), b->stream);
    for (auto& kv : b->bra_by_class) {
        if (!fast3c_supported(kv.first.first, kv.first.second, 0) || !b->spherical) continue;
        rc |= launch_e_table(kv.first.first, kv.first.second, kv.second, b->d_etab + b->etab_offset[kv.first],
                             b->stream);
        launches++;
    }
    rc |= launch_gen_etabs(b, b->stream, &launches);
    cudaEventRecord(b->events[0], b->stream);
    for (int i = 0; i < n_side; i++) cudaStreamWaitEvent(b->side[i], b->events[0], 0);
    int next = 0;
    for (ClassPlan& pl : b->plans) {
        if (pl.total_items == 0 && pl.total_items32 == 0) continue;
        cudaStream_t s = b->side[next++ % n_side];
        if (pl.fast) {
            if (pl.total_items > 0) {
                BatchMap map = pl.map;
                map.checksum = checksum ? b->d_checksum : nullptr;
                rc |= pl.point ? launch_fast_point(pl.li, pl.lj, pl.bra, pl.ket, map, pl.total_items, b->omega,
                                                   b->d_out, pl.counter, s)
                               : launch_fast3c(pl.li, pl.lj, pl.lk, pl.bra, pl.ket, map, pl.total_items, b->omega,
                                               b->d_out, pl.counter, s);
                launches++;
            }
            if (pl.total_items32 > 0) {
                BatchMap map = pl.map32;
                map.checksum = checksum ? b->d_checksum : nullptr;
                rc |= launch_fast3c(pl.li, pl.lj, pl.lk, pl.bra, pl.ket, map, pl.total_items32, b->omega, b->d_out,
                                    pl.counter32, s, true);
                launches++;
            }
        }
    }
    {
        int n = 0;
        rc |= launch_general_groups(b, checksum, false, nullptr, b->d_out, n);
        launches += n;
    }
    for (int i = 0; i < n_side; i++) {
        cudaEventRecord(b->events[1 + i], b->side[i]);
        cudaStreamWaitEvent(b->stream, b->events[1 + i], 0);
    }
    e = cudaStreamEndCapture(b->stream, &b->graph);
    if (e != cudaSuccess || rc != 0) return fail(b, "graph capture", e);
    if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess) return fail(b, "graph instantiate", e);
    b->launches_per_run = launches;
    return 0;
}

int eip_batch_run(eip_batch* b, int checksum) {
    if (!b || !b->built || !b->d_out) return 2;
    OnDevice on(b);
    if (!on.ok) return fail(b, "cudaSetDevice (batch device)", cudaErrorInvalidDevice);
    if (!b->exec) {
        if (int rc = capture(b, checksum != 0)) return rc;
    }
    cudaError_t e = cudaGraphLaunch(b->exec, b->stream);
    if (e != cudaSuccess) return fail(b, "graph launch", e);
    return 0;
}

int eip_batch_run_class(eip_batch* b, int i_L, int j_L, int k_L) {
    if (!b || !b->built || !b->d_out) return 2;
    OnDevice on(b);
    if (!on.ok) return fail(b, "cudaSetDevice (batch device)", cudaErrorInvalidDevice);
    for (ClassPlan& pl : b->plans) {
        if (pl.li != i_L || pl.lj != j_L || pl.lk != k_L) continue;
        if (pl.total_items == 0 && pl.total_items32 == 0) return 1;
        cudaMemsetAsync(pl.counter, 0, 4 * sizeof(int), b->stream);
        int rc = 0;
        if (!pl.fast) {
            auto et = b->gen_etab_offset.find({pl.li, pl.lj});
            if (et != b->gen_etab_offset.end())
                rc |= launch_general_e_table(pl.li, pl.lj, pl.bra, b->gen_etab_nprim[{pl.li, pl.lj}],
                                             b->d_gen_etab + et->second, b->stream);
            const GenClassSpec sp = gen_spec(b, pl, pl.map, pl.total_items, b->stream);
            rc |= launch_general_multi(&sp, 1, b->spherical, nullptr, b->omega, b->d_out, pl.counter, b->stream);
        }
        else if (pl.total_items > 0)
            rc |= pl.point ? launch_fast_point(pl.li, pl.lj, pl.bra, pl.ket, pl.map, pl.total_items, b->omega,
                                               b->d_out, pl.counter, b->stream)
                           : launch_fast3c(pl.li, pl.lj, pl.lk, pl.bra, pl.ket, pl.map, pl.total_items, b->omega,
                                           b->d_out, pl.counter, b->stream);
        if (pl.fast && pl.total_items32 > 0)
            rc |= launch_fast3c(pl.li, pl.lj, pl.lk, pl.bra, pl.ket, pl.map32, pl.total_items32, b->omega, b->d_out,
                                pl.counter32, b->stream, true);
        return rc == 0 ? 0 : fail(b, "class launch", cudaGetLastError());
    }
    return 1;
}

static size_t win_ob_off(int nm) { return ((sizeof(int) * (4 * nm + 2)) + 7) & ~size_t(7); }

long long eip_batch_window_plan(eip_batch* b, const int* fn_lo, const int* fn_hi, int with_charges) {
    if (!b || !b->built) return -1;
    const int nm = b->n_mol;
    // next slot of the ring; its pinned maps may still be in an earlier upload
    const int slot = b->win_next;
    if (b->win_pending[slot]) {
        cudaError_t e = cudaEventSynchronize(b->win_uploaded[slot]);
        if (e != cudaSuccess) {
            fail(b, "window upload", e);
            return -1;
        }
        b->win_pending[slot] = false;
    }
    void* hw = static_cast<char*>(b->h_win) + b->win_bytes * slot;
    long long total = 0;
    for (ClassPlan& pl : b->plans) {
        int* v = at<int>(hw, pl.win_off);
        int* ib64 = v;
        int* ib32 = v + (nm + 1);
        int* ast = v + 2 * (nm + 1);
        int* acnt = ast + nm;
        long long* ob = at<long long>(hw, pl.win_off + win_ob_off(nm));
        const std::vector<int>& starts = b->ket_start[pl.lk];
        const std::vector<int>& ab = b->ket_aux_begin[pl.lk];
        const int lk = pl.point ? 0 : pl.lk;
        const long long blk_unit = (long long)(b->spherical ? nsph(pl.li) * nsph(pl.lj) * nsph(lk)
                                                            : ncart(pl.li) * ncart(pl.lj) * ncart(lk));
        pl.win_out.assign(nm, 0);
        pl.win_start.assign(nm, 0);
        pl.win_count.assign(nm, 0);
        ib64[0] = ib32[0] = 0;
        for (int m = 0; m < nm; m++) {
            int s0 = ab[m], s1 = ab[m];
            if (!pl.point || with_charges) {
                s0 = ab[m];
                s1 = ab[m + 1];
                if (!pl.point && fn_lo && fn_hi) {
                    s0 = (int)(std::lower_bound(starts.begin() + ab[m], starts.begin() + ab[m + 1], fn_lo[m]) -
                               starts.begin());
                    s1 = (int)(std::lower_bound(starts.begin() + s0, starts.begin() + ab[m + 1], fn_hi[m]) -
                               starts.begin());
                }
            }
            const int cnt = s1 - s0, tiles = pl.fast ? (cnt + 31) / 32 : cnt * pl.gen_chunks;
            ast[m] = s0;
            acnt[m] = cnt;
            ob[m] = total;
            pl.win_out[m] = total;
            pl.win_start[m] = s0;
            pl.win_count[m] = cnt;
            total += (long long)pl.n_sp[m] * cnt * blk_unit;
            const long long i64 = (long long)ib64[m] + (long long)pl.n64[m] * tiles;
            const long long i32 = (long long)ib32[m] + (long long)pl.n32[m] * tiles;
            if (i64 > 0x7fffffffLL || i32 > 0x7fffffffLL) {
                fail(b, "window too large", cudaSuccess);
                return -1;
            }
            ib64[m + 1] = (int)i64;
            ib32[m + 1] = (int)i32;
        }
        pl.win_items64 = ib64[nm];
        pl.win_items32 = ib32[nm];
    }
    b->win_elems = total;
    b->win_slot = slot;
    b->win_next = (slot + 1) % eip_batch::kWinSlots;
    b->win_planned = true;
    b->win_charges = with_charges != 0;
    return total;
}

int eip_batch_window_block(eip_batch* b, int mol, int i_L, int j_L, int k_L, long long* offset, int* n_pair_shells,
                           int* n_aux_shells) {
    if (!b || !b->built || !b->win_planned || mol < 0 || mol >= b->n_mol) return 2;
    for (const ClassPlan& pl : b->plans)
        if (pl.li == i_L && pl.lj == j_L && pl.lk == k_L) {
            *offset = pl.win_out[mol];
            *n_pair_shells = pl.n_sp[mol];
            *n_aux_shells = pl.win_count[mol];
            return 0;
        }
    return 1;
}

int eip_batch_run_window(eip_batch* b, double* device_out, int checksum) {
    if (!b || !b->built || !b->win_planned || !device_out) return 2;
    OnDevice on(b);
    if (!on.ok) return fail(b, "cudaSetDevice (batch device)", cudaErrorInvalidDevice);
    cudaError_t e;
    const int nm = b->n_mol;
    const int n_side = b->n_streams;
    if (b->side.empty()) {
        for (int i = 0; i < n_side; i++) {
            cudaStream_t s;
            if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) return fail(b, "stream", e);
            b->side.push_back(s);
        }
        for (int i = 0; i < 2 * n_side + 1; i++) {
            cudaEvent_t ev;
            if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return fail(b, "event", e);
            b->events.push_back(ev);
        }
    }
    const int slot = b->win_slot;
    void* dw = static_cast<char*>(b->d_win) + b->win_bytes * slot;
    if ((e = cudaMemcpyAsync(dw, static_cast<char*>(b->h_win) + b->win_bytes * slot, b->win_bytes,
                             cudaMemcpyHostToDevice, b->stream)) != cudaSuccess)
        return fail(b, "window upload", e);
    cudaEventRecord(b->win_uploaded[slot], b->stream);
    b->win_pending[slot] = true;
    int rc = 0;
    if (!b->etab_ready) {
        for (auto& kv : b->bra_by_class) {
            if (!fast3c_supported(kv.first.first, kv.first.second, 0) || !b->spherical) continue;
            rc |= launch_e_table(kv.first.first, kv.first.second, kv.second, b->d_etab + b->etab_offset[kv.first],
                                 b->stream);
        }
        rc |= launch_gen_etabs(b, b->stream);
        b->etab_ready = true;
    }
    if (checksum) cudaMemsetAsync(b->d_checksum, 0, sizeof(double) * nm, b->stream);
    cudaEventRecord(b->events[0], b->stream);
    for (int i = 0; i < n_side; i++) cudaStreamWaitEvent(b->side[i], b->events[0], 0);
    int next = 0;
    for (ClassPlan& pl : b->plans) {
        if (pl.win_items64 == 0 && pl.win_items32 == 0) continue;
        cudaStream_t s = b->side[next++ % n_side];
        const int* v = at<int>(dw, pl.win_off);
        const int* ast = v + 2 * (nm + 1);
        const long long* ob = at<long long>(dw, pl.win_off + win_ob_off(nm));
        cudaMemsetAsync(pl.counter, 0, 4 * sizeof(int), s);
        if (pl.fast) {
            if (pl.win_items64 > 0) {
                BatchMap map = pl.map;
                map.item_begin = v;
                map.aux_begin = ast;
                map.aux_count = ast + nm;
                map.out_begin = ob;
                map.checksum = checksum ? b->d_checksum : nullptr;
                rc |= pl.point ? launch_fast_point(pl.li, pl.lj, pl.bra, pl.ket, map, pl.win_items64, b->omega,
                                                   device_out, pl.counter, s)
                               : launch_fast3c(pl.li, pl.lj, pl.lk, pl.bra, pl.ket, map, pl.win_items64, b->omega,
                                               device_out, pl.counter, s);
            }
            if (pl.win_items32 > 0) {
                BatchMap map = pl.map32;
                map.item_begin = v + (nm + 1);
                map.aux_begin = ast;
                map.aux_count = ast + nm;
                map.out_begin = ob;
                map.checksum = checksum ? b->d_checksum : nullptr;
                rc |= launch_fast3c(pl.li, pl.lj, pl.lk, pl.bra, pl.ket, map, pl.win_items32, b->omega, device_out,
                                    pl.counter32, s, true);
            }
        }
    }
    {
        int n = 0;
        rc |= launch_general_groups(b, checksum != 0, true, dw, device_out, n);
    }
    for (int i = 0; i < n_side; i++) {
        cudaEventRecord(b->events[1 + i], b->side[i]);
        cudaStreamWaitEvent(b->stream, b->events[1 + i], 0);
    }
    if (rc != 0) return fail(b, "window launch", cudaGetLastError());
    return 0;
}

int eip_batch_precision_split(eip_batch* b, int i_L, int j_L, int k_L, long long* triplets_fp64,
                              long long* triplets_fp32) {
    if (!b || !b->built) return 2;
    for (const ClassPlan& pl : b->plans)
        if (pl.li == i_L && pl.lj == j_L && pl.lk == k_L) {
            *triplets_fp64 = pl.fast ? pl.triplets64 : 0;
            *triplets_fp32 = pl.fast ? pl.triplets32 : 0;
            if (!pl.fast)
                for (int m = 0; m < b->n_mol; m++) *triplets_fp64 += (long long)pl.n_sp[m] * pl.n_auxsh[m];
            return 0;
        }
    return 1;
}

int eip_batch_upload(eip_batch* b) {
    if (!b || !b->built) return 2;
    cudaError_t e = cudaMemcpyAsync(b->d_tables, b->h_tables, b->table_bytes, cudaMemcpyHostToDevice, b->stream);
    return e == cudaSuccess ? 0 : fail(b, "table upload", e);
}

long long eip_batch_table_bytes(eip_batch* b) { return b && b->built ? (long long)b->table_bytes : -1; }

long long eip_batch_device_bytes(eip_batch* b) { return b && b->built ? (long long)b->device_bytes : -1; }

int eip_batch_class_splits(eip_batch* b, int i_L, int j_L, int k_L) {
    if (!b || !b->built) return -1;
    for (const ClassPlan& pl : b->plans)
        if (pl.li == i_L && pl.lj == j_L && pl.lk == k_L) return pl.fast ? 0 : pl.gen_splits;
    return -1;
}

unsigned long long eip_batch_launches_per_run(eip_batch* b) { return b ? b->launches_per_run : 0; }

int eip_batch_checksums(eip_batch* b, double* host) {
    if (!b || !b->built) return 2;
    cudaError_t e = cudaMemcpyAsync(host, b->d_checksum, sizeof(double) * b->n_mol, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? 0 : fail(b, "checksum copy", e);
}

int eip_batch_sync(eip_batch* b) {
    if (!b || !b->built) return 2;
    cudaError_t e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? 0 : fail(b, "batch kernels", e);
}

int eip_batch_status(eip_batch* b) {
    if (!b || !b->built) return 2;
    for (const ClassPlan& pl : b->plans) {
        int st[4] = {0, 0, 0, 0};
        cudaError_t e = cudaMemcpyAsync(st, pl.counter, sizeof(st), cudaMemcpyDeviceToHost, b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) return fail(b, "status copy", e);
        if (st[1] != 0 || st[3] != 0) {
            snprintf(b->err, sizeof b->err, "class (%d%d|%d) kernel self-check %d/%d", pl.li, pl.lj, pl.lk, st[1], st[3]);
            return 3;
        }
    }
    return 0;
}

void* eip_batch_stream(eip_batch* b) { return b ? (void*)b->stream : nullptr; }

int eip_batch_df_plan(eip_batch* b, const int* n_ao, const int* n_aux) {
    if (!b || !b->built || !n_ao || !n_aux) return 2;
    OnDevice on(b);
    if (!on.ok) return fail(b, "cudaSetDevice (batch device)", cudaErrorInvalidDevice);
    const int nm = b->n_mol;
    b->df_gather_elems = 0;
    std::vector<long long> d_off(nm + 1, 0), g_off(nm + 1, 0);
    for (int m = 0; m < nm; m++) {
        if (n_ao[m] < 0 || n_aux[m] < 0) return fail(b, "df_plan: negative size", cudaSuccess);
        d_off[m + 1] = d_off[m] + (long long)n_ao[m] * n_ao[m];
        g_off[m + 1] = g_off[m] + n_aux[m];
        // every function a block touches must lie inside the molecule's n_ao
        for (auto& kv : b->pairs[m]) {
            const int ni = b->spherical ? nsph(kv.first.first) : ncart(kv.first.first);
            const int nj = b->spherical ? nsph(kv.first.second) : ncart(kv.first.second);
            for (size_t k = 0; k < kv.second.ia.size(); k++)
                if (kv.second.ia[k] < 0 || kv.second.ja[k] < 0 || kv.second.ia[k] + ni > n_ao[m] ||
                    kv.second.ja[k] + nj > n_ao[m])
                    return fail(b, "df_plan: orbital functions beyond n_ao", cudaSuccess);
        }
    }
    std::vector<DfBlock> blocks;
    std::vector<DfGather> gathers;
    std::map<std::pair<int, int>, long long> gather_of;  // (molecule, aux class) -> cg offset
    long long items = 0;
    const int rows_per_item = df_rows_per_item();
    for (const ClassPlan& pl : b->plans) {
        if (pl.point) continue;
        const int ni = b->spherical ? nsph(pl.li) : ncart(pl.li), nj = b->spherical ? nsph(pl.lj) : ncart(pl.lj),
                  nk = b->spherical ? nsph(pl.lk) : ncart(pl.lk);
        const BraTable& bra = b->bra_by_class[{pl.li, pl.lj}];
        for (int m = 0; m < nm; m++) {
            if (pl.n_sp[m] == 0 || pl.n_auxsh[m] == 0) continue;
            DfBlock bk{};
            bk.out_off = pl.out_begin[m];
            bk.d_off = d_off[m];
            bk.g_off = g_off[m];
            bk.ao = bra.grp_ao + pl.sp0[m];
            bk.aux_start = pl.ket.grp_start + pl.aux0[m];
            auto git = gather_of.find({m, pl.lk});
            if (git == gather_of.end()) {
                const long long off = b->df_gather_elems;
                gathers.push_back(DfGather{off, g_off[m], bk.aux_start, nk, pl.n_auxsh[m], off});
                b->df_gather_elems += (long long)nk * pl.n_auxsh[m];
                git = gather_of.emplace(std::make_pair(m, pl.lk), off).first;
            }
            bk.cg_off = git->second;
            bk.nsp = pl.n_sp[m];
            bk.ni = ni;
            bk.nj = nj;
            bk.nk = nk;
            bk.nax = pl.n_auxsh[m];
            bk.n_ao = n_ao[m];
            bk.item0 = (int)items;
            const std::vector<int>& starts = b->ket_start[pl.lk];
            if (starts[pl.aux0[m] + pl.n_auxsh[m] - 1] + nk > n_aux[m])
                return fail(b, "df_plan: auxiliary functions beyond n_aux", cudaSuccess);
            items += ((long long)bk.nsp * ni * nj + rows_per_item - 1) / rows_per_item;
            if (items > 0x7fffffffLL) return fail(b, "df_plan: too many work items", cudaSuccess);
            blocks.push_back(bk);
        }
    }
    cudaError_t e;
    if (b->d_df) cudaFree(b->d_df);
    b->d_df = nullptr;
    if ((e = cudaMalloc((void**)&b->d_df, sizeof(DfBlock) * std::max<size_t>(blocks.size(), 1))) != cudaSuccess)
        return fail(b, "df_plan: block list", e);
    if (!blocks.empty() &&
        (e = cudaMemcpy(b->d_df, blocks.data(), sizeof(DfBlock) * blocks.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(b, "df_plan: block list upload", e);
    if (b->d_dfg) cudaFree(b->d_dfg);
    if (b->d_cg) cudaFree(b->d_cg);
    b->d_dfg = nullptr;
    b->d_cg = nullptr;
    if ((e = cudaMalloc((void**)&b->d_dfg, sizeof(DfGather) * std::max<size_t>(gathers.size(), 1))) != cudaSuccess ||
        (e = cudaMalloc((void**)&b->d_cg, sizeof(double) * std::max<long long>(b->df_gather_elems, 1))) != cudaSuccess)
        return fail(b, "df_plan: gathered vectors", e);
    if (!gathers.empty() && (e = cudaMemcpy(b->d_dfg, gathers.data(), sizeof(DfGather) * gathers.size(),
                                            cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(b, "df_plan: gather list upload", e);
    b->df_gathers = (int)gathers.size();
    b->df_blocks = (int)blocks.size();
    b->df_items = (int)items;
    b->df_ao2 = d_off[nm];
    b->df_aux = g_off[nm];
    return 0;
}

int eip_batch_df_gamma(eip_batch* b, const double* D, double* gamma) {
    if (!b || !b->built || !b->d_out || !b->d_df || !D || !gamma) return 2;
    OnDevice on(b);
    if (!on.ok) return fail(b, "cudaSetDevice (batch device)", cudaErrorInvalidDevice);
    cudaError_t e = cudaMemsetAsync(gamma, 0, sizeof(double) * b->df_aux, b->stream);
    if (e != cudaSuccess) return fail(b, "df_gamma: clear", e);
    if (launch_df_gamma(b->d_df, b->df_blocks, b->df_items, b->d_out, D, gamma, b->stream) != 0)
        return fail(b, "df_gamma launch", cudaGetLastError());
    return 0;
}

int eip_batch_df_coulomb(eip_batch* b, const double* c, double* J) {
    if (!b || !b->built || !b->d_out || !b->d_df || !c || !J) return 2;
    OnDevice on(b);
    if (!on.ok) return fail(b, "cudaSetDevice (batch device)", cudaErrorInvalidDevice);
    cudaError_t e = cudaMemsetAsync(J, 0, sizeof(double) * b->df_ao2, b->stream);
    if (e != cudaSuccess) return fail(b, "df_coulomb: clear", e);
    if (launch_df_coulomb(b->d_df, b->df_blocks, b->df_items, b->d_dfg, b->df_gathers, b->df_gather_elems, b->d_cg,
                          b->d_out, c, J, b->stream) != 0)
        return fail(b, "df_coulomb launch", cudaGetLastError());
    return 0;
}

int eip_batch_copy_output(eip_batch* b, long long offset, long long count, double* host) {
    if (!b || !b->built || !b->d_out || offset < 0 || count < 0 || offset + count > b->out_elems) return 2;
    cudaError_t e = cudaMemcpyAsync(host, b->d_out + offset, sizeof(double) * count, cudaMemcpyDeviceToHost,
                                    b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? 0 : fail(b, "output copy", e);
}

void eip_batch_destroy(eip_batch* b) {
    if (!b) return;
    OnDevice on(b);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->own_out && b->d_out) cudaFree(b->d_out);
    if (b->d_tables) cudaFree(b->d_tables);
    if (b->h_tables) cudaFreeHost(b->h_tables);
    if (b->d_etab) cudaFree(b->d_etab);
    if (b->d_checksum) cudaFree(b->d_checksum);
    if (b->d_df) cudaFree(b->d_df);
    if (b->d_dfg) cudaFree(b->d_dfg);
    if (b->d_cg) cudaFree(b->d_cg);
    if (b->d_gen) cudaFree(b->d_gen);
    if (b->d_split) cudaFree(b->d_split);
    if (b->d_gen_etab) cudaFree(b->d_gen_etab);
    if (b->d_arrive) cudaFree(b->d_arrive);
    if (b->d_win) cudaFree(b->d_win);
    if (b->h_win) cudaFreeHost(b->h_win);
    for (auto ev : b->win_uploaded)
        if (ev) cudaEventDestroy(ev);
    for (auto s : b->side) cudaStreamDestroy(s);
    for (auto ev : b->events) cudaEventDestroy(ev);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

}  // extern "C"
