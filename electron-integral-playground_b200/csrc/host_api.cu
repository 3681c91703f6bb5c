// C ABI of libmolecular_integral.so: the reference's four entry points
// (drop-in) plus the eip_* extensions.  Host code only; kernels live in the
// other translation units.
//
// Per legacy call (one angular class, host buffers, output accumulated with
// +=, as MI/*.cpp do):
//   1. group the primitive pairs by contracted shell pair (i_ao_start,
//      j_ao_start) and the auxiliary primitives by shell, and pack the device
//      tables into a reusable pinned staging buffer;
//   2. one H2D copy, then the fast templated kernel (common classes) or the
//      generic kernel + transform, which write the class's contracted blocks
//      in a compact device layout (each element once, no atomics);
//   3. one D2H copy of the compact blocks, and a multi-threaded scatter-add
//      into the caller's dense array, mirrored like the reference
//      (MI/three_center.cpp:242-244).
// The caller's output array is never copied to or from the device.
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <numeric>
#include <vector>

#include "eip_common.cuh"
#include "eip_internal.h"
#include "../../include/eip_b200.h"

namespace eip {

thread_local char g_last_error[512] = "";

void set_error(const char* what, cudaError_t e) {
    if (e == cudaSuccess) snprintf(g_last_error, sizeof g_last_error, "%s", what);
    else snprintf(g_last_error, sizeof g_last_error, "%s: %s", what, cudaGetErrorString(e));
    fprintf(stderr, "[eip] %s\n", g_last_error);
}

namespace {

struct DeviceBuffer {
    void* ptr = nullptr;
    size_t size = 0;
    cudaError_t reserve(size_t bytes) {
        if (bytes <= size) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        size = 0;
        size_t want = std::max(bytes, size_t(1) << 20);
        cudaError_t e = cudaMalloc(&ptr, want);
        if (e == cudaSuccess) size = want;
        return e;
    }
};

struct PinnedBuffer {
    void* ptr = nullptr;
    size_t size = 0;
    cudaError_t reserve(size_t bytes) {
        if (bytes <= size) return cudaSuccess;
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        size = 0;
        size_t want = std::max(bytes + bytes / 4, size_t(1) << 20);
        cudaError_t e = cudaMallocHost(&ptr, want);
        if (e == cudaSuccess) size = want;
        return e;
    }
};

struct Context {
    std::mutex mu;
    int device = -1;
    cudaStream_t stream = nullptr;
    PinnedBuffer h_in, h_out;
    DeviceBuffer d_in, d_raw, d_out, d_etab, d_misc;
    unsigned long long launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_kernel_ms = 0.0f;  // device time of the last class's kernels
};

Context& ctx() {
    static Context c;
    return c;
}

// The reference-ABI calls run on the library context's device (the one
// current at eip_init or at the first call), whatever device the calling
// thread has current; the caller's device is restored on return.
struct DeviceGuard {
    int saved = -1;
    bool switched = false;
    cudaError_t enter(int dev) {
        cudaError_t e = cudaGetDevice(&saved);
        if (e != cudaSuccess) return e;
        if (saved == dev) return cudaSuccess;
        e = cudaSetDevice(dev);
        switched = e == cudaSuccess;
        return e;
    }
    ~DeviceGuard() {
        if (switched) cudaSetDevice(saved);
    }
};

int ensure_context_locked(Context& c, DeviceGuard* guard = nullptr) {
    if (c.device >= 0) {
        if (guard) {
            cudaError_t e = guard->enter(c.device);
            if (e != cudaSuccess) {
                set_error("cudaSetDevice (library context device)", e);
                return 2;
            }
        }
        return 0;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev >= kMaxDevices) {
        set_error("no usable CUDA device", e);
        return 2;
    }
    e = cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        set_error("cudaStreamCreate", e);
        return 2;
    }
    if (cudaEventCreate(&c.ev0) != cudaSuccess || cudaEventCreate(&c.ev1) != cudaSuccess) {
        set_error("cudaEventCreate", cudaGetLastError());
        return 2;
    }
    if (int rc = ensure_device_tables()) {
        set_error("constant table upload", (cudaError_t)rc);
        return 2;
    }
    c.device = dev;
    return 0;
}

// Byte layout of several arrays in one staging buffer (256-byte aligned).
struct Layout {
    size_t total = 0;
    size_t add(size_t bytes) {
        size_t off = total;
        total += (bytes + 255) & ~size_t(255);
        return off;
    }
};

// Host-side grouping of primitive pairs by contracted shell pair.
struct PairGroups {
    std::vector<int> order;   // primitive index in grouped order
    std::vector<int> begin;   // n_group + 1
    std::vector<int> ao_i, ao_j;
};

PairGroups group_pairs(const int* ia, const int* ja, int n) {
    PairGroups g;
    g.order.resize(n);
    std::iota(g.order.begin(), g.order.end(), 0);
    std::stable_sort(g.order.begin(), g.order.end(), [&](int x, int y) {
        return ia[x] != ia[y] ? ia[x] < ia[y] : ja[x] < ja[y];
    });
    for (int k = 0; k < n; k++) {
        int p = g.order[k];
        if (k == 0 || ia[p] != g.ao_i.back() || ja[p] != g.ao_j.back()) {
            g.begin.push_back(k);
            g.ao_i.push_back(ia[p]);
            g.ao_j.push_back(ja ? ja[p] : 0);
        }
    }
    g.begin.push_back(n);
    return g;
}

PairGroups group_one(const int* start, int n) {
    std::vector<int> zeros(n, 0);
    PairGroups g = group_pairs(start, zeros.data(), n);
    return g;
}

// Pinned staging -> device, returns device tables.
struct Staged {
    BraTable bra{};
    KetTable ket{};
    const double* prim_b = nullptr;
    int n_bra_prims = 0;
};

template <typename T>
T* at(void* base, size_t off) {
    return reinterpret_cast<T*>(static_cast<char*>(base) + off);
}

// kind: 0 pair bra (P, A, B arrays), 1 one-centre bra (aux A array)
struct BraInput {
    int kind;
    const double* P;
    const double* A;
    const double* B;
    const double* coef;
    const int* ia;
    const int* ja;
    int n;
};
struct KetInput {
    int kind;  // 0 aux shells, 1 point charges (xyz rows)
    const double* C;
    const double* coef;
    const int* start;
    int n;
};

int stage_inputs(Context& c, const BraInput& bi, const KetInput& ki, Staged& st, PairGroups& bg, PairGroups& kg) {
    bg = bi.kind == 0 ? group_pairs(bi.ia, bi.ja, bi.n) : group_one(bi.ia, bi.n);
    const int nb = (int)bg.ao_i.size(), npb = bi.n;
    int nk = 0, npk = 0;
    if (ki.n > 0) {
        if (ki.kind == 0) {
            kg = group_one(ki.start, ki.n);
            nk = (int)kg.ao_i.size();
        } else {
            kg.order.resize(ki.n);
            std::iota(kg.order.begin(), kg.order.end(), 0);
            kg.begin.resize(ki.n + 1);
            std::iota(kg.begin.begin(), kg.begin.end(), 0);
            kg.ao_i.resize(ki.n);
            std::iota(kg.ao_i.begin(), kg.ao_i.end(), 0);
            nk = ki.n;
        }
        npk = ki.n;
    }
    Layout L;
    const size_t o_bbeg = L.add(sizeof(int) * (nb + 1)), o_bao = L.add(sizeof(int2) * nb),
                 o_bab = L.add(sizeof(double4) * nb), o_bp = L.add(sizeof(double4) * npb),
                 o_bpa = L.add(sizeof(double4) * npb), o_bb = L.add(sizeof(double) * npb);
    const size_t o_kbeg = L.add(sizeof(int) * (nk + 1)), o_kst = L.add(sizeof(int) * nk),
                 o_kc = L.add(sizeof(double4) * npk), o_kco = L.add(sizeof(double) * npk);
    cudaError_t e = c.h_in.reserve(L.total);
    if (e == cudaSuccess) e = c.d_in.reserve(L.total);
    if (e != cudaSuccess) {
        set_error("staging allocation", e);
        return 2;
    }
    void* h = c.h_in.ptr;
    memcpy(at<int>(h, o_bbeg), bg.begin.data(), sizeof(int) * (nb + 1));
    for (int g = 0; g < nb; g++) {
        at<int2>(h, o_bao)[g] = make_int2(bg.ao_i[g], bg.ao_j[g]);
        const int p = bg.order[bg.begin[g]];
        at<double4>(h, o_bab)[g] = bi.kind == 0 ? make_double4(bi.A[4 * p] - bi.B[4 * p], bi.A[4 * p + 1] - bi.B[4 * p + 1],
                                                               bi.A[4 * p + 2] - bi.B[4 * p + 2], 0.0)
                                                : make_double4(0.0, 0.0, 0.0, 0.0);
    }
    for (int k = 0; k < npb; k++) {
        const int p = bg.order[k];
        if (bi.kind == 0) {
            const double* P = bi.P + 4 * p;
            const double* A = bi.A + 4 * p;
            at<double4>(h, o_bp)[k] = make_double4(P[0], P[1], P[2], P[3]);
            at<double4>(h, o_bpa)[k] = make_double4(P[0] - A[0], P[1] - A[1], P[2] - A[2], bi.coef[p]);
            at<double>(h, o_bb)[k] = bi.B ? bi.B[4 * p + 3] : 0.0;
        } else {
            const double* A = bi.A + 4 * p;
            at<double4>(h, o_bp)[k] = make_double4(A[0], A[1], A[2], A[3]);
            at<double4>(h, o_bpa)[k] = make_double4(0.0, 0.0, 0.0, bi.coef[p]);
            at<double>(h, o_bb)[k] = 0.0;
        }
    }
    if (nk > 0) {
        memcpy(at<int>(h, o_kbeg), kg.begin.data(), sizeof(int) * (nk + 1));
        for (int g = 0; g < nk; g++) at<int>(h, o_kst)[g] = kg.ao_i[g];
        for (int k = 0; k < npk; k++) {
            const int p = kg.order[k];
            if (ki.kind == 0) {
                const double* C = ki.C + 4 * p;
                at<double4>(h, o_kc)[k] = make_double4(C[0], C[1], C[2], C[3]);
                at<double>(h, o_kco)[k] = ki.coef[p];
            } else {
                const double* C = ki.C + 3 * p;
                at<double4>(h, o_kc)[k] = make_double4(C[0], C[1], C[2], 0.0);
                at<double>(h, o_kco)[k] = 1.0;
            }
        }
    }
    e = cudaMemcpyAsync(c.d_in.ptr, h, L.total, cudaMemcpyHostToDevice, c.stream);
    if (e != cudaSuccess) {
        set_error("H2D copy", e);
        return 2;
    }
    void* d = c.d_in.ptr;
    st.bra = BraTable{nb, at<int>(d, o_bbeg), at<int2>(d, o_bao), at<double4>(d, o_bab), at<double4>(d, o_bp),
                      at<double4>(d, o_bpa), nullptr};
    st.n_bra_prims = npb;
    st.prim_b = at<double>(d, o_bb);
    st.ket = KetTable{nk, at<int>(d, o_kbeg), at<int>(d, o_kst), at<double4>(d, o_kc), at<double>(d, o_kco)};
    return 0;
}

// Computes the compact block of one class into c.d_out and copies it to c.h_out.
// mode: 0 three-centre, 1 two-centre (the bra is the one-centre pair class
// (0, l_P): A = B = P), 2 nuclear attraction (point-charge ket), 3 overlap.
// Three-centre, two-centre and nuclear attraction run as a batch of one
// molecule: the fast kernel of the class when there is one (spherical output,
// pair class l_i <= l_j <= 2 or (0, 3), (0, 4), ket l <= 4), else the general
// kernel; both write the packed block [pair][I][J][K][ket shell].
int compute_class(Context& c, int mode, int li, int lj, int lk, bool spherical, double omega, const Staged& st,
                  size_t n_out) {
    cudaError_t e = c.d_out.reserve(sizeof(double) * n_out);
    if (e == cudaSuccess) e = c.h_out.reserve(sizeof(double) * n_out);
    if (e != cudaSuccess) {
        set_error("output allocation", e);
        return 2;
    }
    int rc = 0;
    double* dout = static_cast<double*>(c.d_out.ptr);
    const int n_bra = st.bra.n_group, n_ket = mode == 3 ? 1 : st.ket.n_group;
    cudaEventRecord(c.ev0, c.stream);
    if (mode == 3) {
        const size_t n_raw = (size_t)n_bra * ncart(li) * ncart(lj);
        e = c.d_raw.reserve(sizeof(double) * n_raw);
        if (e != cudaSuccess) {
            set_error("scratch allocation", e);
            return 2;
        }
        double* raw = static_cast<double*>(c.d_raw.ptr);
        rc = launch_overlap_raw(li, lj, st.bra, st.prim_b, raw, c.stream);
        if (rc == 0) rc = launch_transform(li, lj, 0, spherical, n_bra, 1, raw, dout, c.stream);
        c.launches += 2;
        if (rc != 0) {
            set_error("kernel launch", cudaGetLastError());
            return 2;
        }
    } else {
        const bool point = mode == 2;
        const bool fast = spherical && fast3c_supported(li, lj, point ? 0 : lk);
        const long long items = fast ? (long long)n_bra * ((n_ket + 31) / 32)
                                     : (long long)n_bra * n_ket * general_chunks(li, lj, lk, point, spherical);
        if (items > 0x7fffffffLL) {
            set_error("class too large for one call", cudaSuccess);
            return 2;
        }
        e = c.d_misc.reserve(256);
        if (e == cudaSuccess && fast)
            e = c.d_etab.reserve(sizeof(double) * e_table_doubles(li, lj) * (size_t)st.n_bra_prims);
        if (e != cudaSuccess) {
            set_error("work-list allocation", e);
            return 2;
        }
        // one-molecule work map: [0..1] counter/status, [4..5] item_begin,
        // [8..9] pair begin, [12..13] ket begin, then out_begin (= 0)
        int* misc = static_cast<int*>(c.d_misc.ptr);
        const int host_misc[16] = {0, 0, 0, 0, 0, (int)items, 0, 0, 0, n_bra, 0, 0, 0, n_ket, 0, 0};
        cudaMemcpyAsync(misc, host_misc, sizeof(host_misc), cudaMemcpyHostToDevice, c.stream);
        long long* out_begin = reinterpret_cast<long long*>(misc + 16);
        cudaMemsetAsync(out_begin, 0, sizeof(long long), c.stream);
        BatchMap map{1, misc + 4, misc + 8, misc + 12, out_begin, nullptr, nullptr, nullptr};
        if (fast) {
            BraTable bra = st.bra;
            bra.prim_E = static_cast<double*>(c.d_etab.ptr);
            rc = launch_e_table(li, lj, bra, static_cast<double*>(c.d_etab.ptr), c.stream);
            if (rc == 0)
                rc = point ? launch_fast_point(li, lj, bra, st.ket, map, (int)items, omega, dout, misc, c.stream)
                           : launch_fast3c(li, lj, lk, bra, st.ket, map, (int)items, omega, dout, misc, c.stream);
            c.launches += 2;
        } else {
            rc = launch_general(li, lj, lk, point, spherical, st.bra, st.ket, map, (int)items, omega, dout, misc,
                                c.stream);
            c.launches += 1;
        }
        if (rc != 0) {
            set_error(rc == 3 ? "class needs more shared memory than a CTA has" : "kernel launch",
                      cudaGetLastError());
            return 2;
        }
        int status[2] = {0, 0};
        e = cudaMemcpyAsync(status, misc, sizeof(status), cudaMemcpyDeviceToHost, c.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
        if (e != cudaSuccess || status[1] != 0) {
            snprintf(g_last_error, sizeof g_last_error, "integral kernel self-check %d (cuda: %s)", status[1],
                     cudaGetErrorString(e));
            fprintf(stderr, "[eip] %s\n", g_last_error);
            return 2;
        }
    }
    cudaEventRecord(c.ev1, c.stream);
    e = cudaMemcpyAsync(c.h_out.ptr, dout, sizeof(double) * n_out, cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    if (e == cudaSuccess) cudaEventElapsedTime(&c.last_kernel_ms, c.ev0, c.ev1);
    if (e != cudaSuccess) {
        set_error("integral kernels", e);
        return 2;
    }
    return 0;
}

int unsupported(const char* fn, int i_L, int j_L, int k_L, bool has_k) {
    if (has_k)
        printf("%s function does not support angular i_L = %d, j_L = %d, k_L = %d\n", fn, i_L, j_L, k_L);
    else
        printf("%s function does not support angular i_L = %d, j_L = %d\n", fn, i_L, j_L);
    fflush(stdout);
    return 1;
}

}  // namespace
}  // namespace eip

using namespace eip;

extern "C" {

int eip_init(int device) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lock(c.mu);
    if (device >= 0 && c.device < 0) {
        cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) {
            set_error("cudaSetDevice", e);
            return 2;
        }
    }
    return ensure_context_locked(c);
}

const char* eip_last_error(void) { return g_last_error; }

unsigned long long eip_kernel_launch_count(void) { return ctx().launches; }

float eip_last_kernel_ms(void) { return ctx().last_kernel_ms; }

int eip_tune_set(int i_L, int j_L, int k_L, int variant) { return fast3c_set_variant(i_L, j_L, k_L, variant); }

int eip_tune_get(int i_L, int j_L, int k_L) { return fast3c_variant(i_L, j_L, k_L); }

int eip_tune_set_fp32(int i_L, int j_L, int k_L, int variant) {
    return fast3c_set_variant_fp32(i_L, j_L, k_L, variant);
}

int eip_tune_get_fp32(int i_L, int j_L, int k_L) { return fast3c_variant_fp32(i_L, j_L, k_L); }

int eip_boys(int L, const double* T, int n, double* F) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lock(c.mu);
    DeviceGuard guard;
    if (int rc = ensure_context_locked(c, &guard)) return rc;
    if (L < 0 || L > kMaxBoysM) return 1;
    if (n <= 0) return 0;
    const size_t out_bytes = sizeof(double) * (size_t)n * (L + 1);
    cudaError_t e = c.d_in.reserve(sizeof(double) * n);
    if (e == cudaSuccess) e = c.d_out.reserve(out_bytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c.d_in.ptr, T, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream);
    if (e != cudaSuccess) {
        set_error("eip_boys staging", e);
        return 2;
    }
    if (launch_boys_probe(L, (const double*)c.d_in.ptr, n, (double*)c.d_out.ptr, c.stream)) return 2;
    c.launches += 1;
    e = cudaMemcpyAsync(F, c.d_out.ptr, out_bytes, cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess) {
        set_error("eip_boys", e);
        return 2;
    }
    return 0;
}

int three_center(const int i_L, const int j_L, const int k_L, const double* pair_P_p, const double* pair_A_a,
                 const double* pair_B_b, const double* pair_coefficient, const int* pair_i_ao_start,
                 const int* pair_j_ao_start, const int n_pair_ij, const double* aux_A_a,
                 const double* aux_coefficient, const int* aux_i_aux_start, const int n_aux_primitive_k,
                 double* J3c_matrix, const int n_ao, const int n_aux, const bool spherical, const double omega) {
    (void)n_aux;
    if (i_L < 0 || j_L < 0 || k_L < 0 || i_L > j_L || j_L > kMaxOrbitalL || k_L > kMaxAuxL)
        return unsupported(__func__, i_L, j_L, k_L, true);
    if (n_pair_ij <= 0 || n_aux_primitive_k <= 0) return 0;
    Context& c = ctx();
    std::lock_guard<std::mutex> lock(c.mu);
    DeviceGuard guard;
    if (int rc = ensure_context_locked(c, &guard)) return rc;
    Staged st;
    PairGroups bg, kg;
    BraInput bi{0, pair_P_p, pair_A_a, pair_B_b, pair_coefficient, pair_i_ao_start, pair_j_ao_start, n_pair_ij};
    KetInput ki{0, aux_A_a, aux_coefficient, aux_i_aux_start, n_aux_primitive_k};
    if (int rc = stage_inputs(c, bi, ki, st, bg, kg)) return rc;
    const int ni = spherical ? nsph(i_L) : ncart(i_L), nj = spherical ? nsph(j_L) : ncart(j_L),
              nk = spherical ? nsph(k_L) : ncart(k_L);
    const int nb = st.bra.n_group, nkt = st.ket.n_group;
    const size_t n_out = (size_t)nb * ni * nj * nk * nkt;
    if (int rc = compute_class(c, 0, i_L, j_L, k_L, spherical, omega, st, n_out)) return rc;
    const double* h = static_cast<const double*>(c.h_out.ptr);
    const size_t nao = (size_t)n_ao, nao2 = nao * nao;
#pragma omp parallel for schedule(dynamic, 16)
    for (int b = 0; b < nb; b++) {
        const size_t i0 = (size_t)bg.ao_i[b], j0 = (size_t)bg.ao_j[b];
        const bool mirror = i0 != j0;
        for (int I = 0; I < ni; I++)
            for (int J = 0; J < nj; J++)
                for (int K = 0; K < nk; K++) {
                    const double* row = h + ((((size_t)b * ni + I) * nj + J) * nk + K) * nkt;
                    for (int a = 0; a < nkt; a++) {
                        const size_t k0 = (size_t)kg.ao_i[a] + K;
                        J3c_matrix[k0 * nao2 + (i0 + I) * nao + (j0 + J)] += row[a];
                        if (mirror) J3c_matrix[k0 * nao2 + (j0 + J) * nao + (i0 + I)] += row[a];
                    }
                }
    }
    return 0;
}

int two_center(const int i_L, const int j_L, const double* aux_A_a, const double* aux_i_coefficient,
               const int* aux_i_aux_start, const int n_aux_primitive_i, const double* aux_B_b,
               const double* aux_j_coefficient, const int* aux_j_aux_start, const int n_aux_primitive_j,
               double* J2c_matrix, const int n_aux, const bool spherical, const double omega) {
    if (i_L < 0 || j_L < 0 || i_L > j_L || j_L > kMaxAuxL) return unsupported(__func__, i_L, j_L, 0, false);
    if (n_aux_primitive_i <= 0 || n_aux_primitive_j <= 0) return 0;
    Context& c = ctx();
    std::lock_guard<std::mutex> lock(c.mu);
    DeviceGuard guard;
    if (int rc = ensure_context_locked(c, &guard)) return rc;
    Staged st;
    PairGroups bg, kg;
    BraInput bi{1, nullptr, aux_A_a, nullptr, aux_i_coefficient, aux_i_aux_start, nullptr, n_aux_primitive_i};
    KetInput ki{0, aux_B_b, aux_j_coefficient, aux_j_aux_start, n_aux_primitive_j};
    if (int rc = stage_inputs(c, bi, ki, st, bg, kg)) return rc;
    const int ni = spherical ? nsph(i_L) : ncart(i_L), nk = spherical ? nsph(j_L) : ncart(j_L);
    const int nb = st.bra.n_group, nkt = st.ket.n_group;
    const size_t n_out = (size_t)nb * ni * nk * nkt;
    // reference skip: same class and i_aux_start > j_aux_start (MI/two_center.cpp:136-138);
    // every block is computed, the skipped ones are not scattered
    const int skip = i_L == j_L ? 1 : 0;
    if (int rc = compute_class(c, 1, 0, i_L, j_L, spherical, omega, st, n_out)) return rc;
    const double* h = static_cast<const double*>(c.h_out.ptr);
    const size_t na = (size_t)n_aux;
#pragma omp parallel for schedule(dynamic, 8)
    for (int b = 0; b < nb; b++) {
        const size_t i0 = (size_t)bg.ao_i[b];
        for (int I = 0; I < ni; I++)
            for (int K = 0; K < nk; K++) {
                const double* row = h + (((size_t)b * ni + I) * nk + K) * nkt;
                for (int a = 0; a < nkt; a++) {
                    const size_t j0 = (size_t)kg.ao_i[a];
                    if (skip && i0 > j0) continue;
                    J2c_matrix[(i0 + I) * na + (j0 + K)] += row[a];
                    if (i0 != j0) J2c_matrix[(j0 + K) * na + (i0 + I)] += row[a];
                }
            }
    }
    return 0;
}

int nuclear_attraction(const int i_L, const int j_L, const double* pair_P_p, const double* pair_A_a,
                       const double* pair_B_b, const double* pair_coefficient, const int* pair_i_ao_start,
                       const int* pair_j_ao_start, const int n_pair, const double* charge_position,
                       const int n_charge, double* V_tensor, const int n_ao, const bool spherical,
                       const double omega) {
    if (i_L < 0 || j_L < 0 || i_L > j_L || j_L > kMaxOrbitalL) return unsupported(__func__, i_L, j_L, 0, false);
    if (n_pair <= 0 || n_charge <= 0) return 0;
    Context& c = ctx();
    std::lock_guard<std::mutex> lock(c.mu);
    DeviceGuard guard;
    if (int rc = ensure_context_locked(c, &guard)) return rc;
    Staged st;
    PairGroups bg, kg;
    BraInput bi{0, pair_P_p, pair_A_a, pair_B_b, pair_coefficient, pair_i_ao_start, pair_j_ao_start, n_pair};
    KetInput ki{1, charge_position, nullptr, nullptr, n_charge};
    if (int rc = stage_inputs(c, bi, ki, st, bg, kg)) return rc;
    const int ni = spherical ? nsph(i_L) : ncart(i_L), nj = spherical ? nsph(j_L) : ncart(j_L);
    const int nb = st.bra.n_group, nc = n_charge;
    const size_t n_out = (size_t)nb * ni * nj * nc;
    if (int rc = compute_class(c, 2, i_L, j_L, 0, spherical, omega, st, n_out)) return rc;
    const double* h = static_cast<const double*>(c.h_out.ptr);
    const size_t nao = (size_t)n_ao;
#pragma omp parallel for schedule(dynamic, 16)
    for (int b = 0; b < nb; b++) {
        const size_t i0 = (size_t)bg.ao_i[b], j0 = (size_t)bg.ao_j[b];
        for (int I = 0; I < ni; I++)
            for (int J = 0; J < nj; J++) {
                const double* row = h + (((size_t)b * ni + I) * nj + J) * nc;
                double* dst = V_tensor + ((i0 + I) * nao + (j0 + J)) * nc;
                for (int q = 0; q < nc; q++) dst[q] += row[q];
                if (i0 != j0) {
                    double* mir = V_tensor + ((j0 + J) * nao + (i0 + I)) * nc;
                    for (int q = 0; q < nc; q++) mir[q] += row[q];
                }
            }
    }
    return 0;
}

int overlap(const int i_L, const int j_L, const double* pair_A_a, const double* pair_B_b,
            const double* pair_coefficient, const int* pair_i_ao_start, const int* pair_j_ao_start, const int n_pair,
            double* S_matrix, const int n_ao, const bool spherical) {
    if (i_L < 0 || j_L < 0 || i_L > j_L || j_L > kMaxOrbitalL) return unsupported(__func__, i_L, j_L, 0, false);
    if (n_pair <= 0) return 0;
    Context& c = ctx();
    std::lock_guard<std::mutex> lock(c.mu);
    DeviceGuard guard;
    if (int rc = ensure_context_locked(c, &guard)) return rc;
    // The overlap entry carries no P_p: rebuild (P, p) rows from A and B.
    std::vector<double> P(4 * (size_t)n_pair);
    for (int k = 0; k < n_pair; k++) {
        const double* A = pair_A_a + 4 * k;
        const double* B = pair_B_b + 4 * k;
        const double p = A[3] + B[3];
        for (int d = 0; d < 3; d++) P[4 * k + d] = (A[3] * A[d] + B[3] * B[d]) / p;
        P[4 * k + 3] = p;
    }
    Staged st;
    PairGroups bg, kg;
    BraInput bi{0, P.data(), pair_A_a, pair_B_b, pair_coefficient, pair_i_ao_start, pair_j_ao_start, n_pair};
    KetInput ki{0, nullptr, nullptr, nullptr, 0};
    if (int rc = stage_inputs(c, bi, ki, st, bg, kg)) return rc;
    const int ni = spherical ? nsph(i_L) : ncart(i_L), nj = spherical ? nsph(j_L) : ncart(j_L);
    const int nb = st.bra.n_group;
    const size_t n_out = (size_t)nb * ni * nj;
    if (int rc = compute_class(c, 3, i_L, j_L, 0, spherical, 0.0, st, n_out)) return rc;
    const double* h = static_cast<const double*>(c.h_out.ptr);
    const size_t nao = (size_t)n_ao;
    for (int b = 0; b < nb; b++) {
        const size_t i0 = (size_t)bg.ao_i[b], j0 = (size_t)bg.ao_j[b];
        for (int I = 0; I < ni; I++)
            for (int J = 0; J < nj; J++) {
                const double v = h[((size_t)b * ni + I) * nj + J];
                S_matrix[(i0 + I) * nao + (j0 + J)] += v;
                if (i0 != j0) S_matrix[(j0 + J) * nao + (i0 + I)] += v;
            }
    }
    return 0;
}

}  // extern "C"
