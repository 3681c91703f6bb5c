// Screened primitive shell-pair tables built on the device: the reference
// front end's form_pair_data (pair_utility.py:6-188) as kernels.
//
// Per (l_i, l_j) class: the shell pairs in the reference's loop order (i shell
// outer, j shell inner, l_i < l_j or equal l with i_ao_start <= j_ao_start);
// one thread per shell pair evaluates the upper bound of each of its
// primitive pairs with the reference's sequence of operations (the distance
// is decremented cumulatively over the primitive loops and clamped after each
// ket primitive), keeps those with bound >= threshold, and the kept pairs are
// stably sorted by descending bound (CUB radix sort, stable) before one more
// kernel writes the structure-of-arrays rows the integral ABI reads.  Products
// and sums that numpy evaluates separately are written with explicit
// round-to-nearest intrinsics so that no multiply-add is fused.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <cub/cub.cuh>
#include <map>
#include <vector>

#include "eip_common.cuh"
#include "eip_internal.h"
#include "../../include/eip_b200.h"

namespace eip {
namespace {

struct ShellRec {
    int l, atom, ao, nprim, prim0;
};

// One shell pair of a class: shells (i, j) and the first of its
// nprim_i * nprim_j candidate slots.
struct PairRec {
    int i, j, slot0;
};

__device__ __forceinline__ double dist3(const double* A, const double* B) {
    const double dx = __dadd_rn(A[0], -B[0]), dy = __dadd_rn(A[1], -B[1]), dz = __dadd_rn(A[2], -B[2]);
    return sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

// Bound of every candidate primitive pair of every shell pair (NaN = rejected).
__global__ void pair_bound_kernel(int n_pair, const PairRec* __restrict__ pairs, const ShellRec* __restrict__ shells,
                                  const double* __restrict__ exps, const double* __restrict__ coefs,
                                  const double* __restrict__ geom, double threshold, double* __restrict__ bound) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_pair) return;
    const PairRec pr = pairs[k];
    const ShellRec si = shells[pr.i], sj = shells[pr.j];
    double d = dist3(geom + 3 * si.atom, geom + 3 * sj.atom);
    const double li = si.l, lj = sj.l;
    const double e = 2.718281828459045;  // numpy's e
    int slot = pr.slot0;
    for (int ip = 0; ip < si.nprim; ip++) {
        const double a = exps[si.prim0 + ip];
        double ca = fabs(coefs[si.prim0 + ip]);
        if (si.l > 0) ca = __dmul_rn(ca, pow(li / __dmul_rn(__dmul_rn(2.0, e), a), li / 2.0));
        d = __dadd_rn(d, -sqrt(li / 2.0 / a));
        for (int jp = 0; jp < sj.nprim; jp++, slot++) {
            const double b = exps[sj.prim0 + jp];
            double cb = fabs(coefs[sj.prim0 + jp]);
            if (sj.l > 0) cb = __dmul_rn(cb, pow(lj / __dmul_rn(__dmul_rn(2.0, e), b), lj / 2.0));
            d = __dadd_rn(d, -sqrt(lj / 2.0 / b));
            d = fmax(d, 0.0);
            const double p = __dadd_rn(a, b);
            const double gauss = exp(__dmul_rn(__dmul_rn(__ddiv_rn(__dmul_rn(-a, b), p), d), d));
            const double cab = __dmul_rn(__dmul_rn(2.0, ca), cb);
            const double ovl = pow(3.141592653589793 / p, 1.5);
            const double sch = __dmul_rn(pow(3.141592653589793 / p, 1.25), pow(2.0, 0.25));
            const double bnd = __dmul_rn(__dmul_rn(cab, gauss), fmax(ovl, sch));
            bound[slot] = bnd < threshold ? __longlong_as_double(0x7ff8000000000000LL) : bnd;
        }
    }
}

__global__ void flag_kernel(int n, const double* __restrict__ bound, int* __restrict__ flag) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) flag[k] = isnan(bound[k]) ? 0 : 1;
}

__global__ void compact_kernel(int n, const double* __restrict__ bound, const int* __restrict__ flag,
                               const int* __restrict__ pos, double* __restrict__ key, int* __restrict__ val) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && flag[k]) {
        key[pos[k]] = bound[k];
        val[pos[k]] = k;
    }
}

// Slot -> (shell pair, ip, jp) by binary search over the pairs' first slots,
// then the reference's row values (pair_utility.py:136-175).
__global__ void pair_rows_kernel(int n_keep, const int* __restrict__ slot_of, int n_pair,
                                 const PairRec* __restrict__ pairs, const ShellRec* __restrict__ shells,
                                 const double* __restrict__ exps, const double* __restrict__ coefs,
                                 const double* __restrict__ geom, double* __restrict__ P_p, double* __restrict__ A_a,
                                 double* __restrict__ B_b, double* __restrict__ coef, int* __restrict__ i_ao,
                                 int* __restrict__ j_ao, int* __restrict__ i_atom, int* __restrict__ j_atom) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_keep) return;
    const int slot = slot_of[r];
    int lo = 0, hi = n_pair - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pairs[mid].slot0 <= slot) lo = mid;
        else hi = mid - 1;
    }
    const PairRec pr = pairs[lo];
    const ShellRec si = shells[pr.i], sj = shells[pr.j];
    const int local = slot - pr.slot0;
    const int ip = local / sj.nprim, jp = local - ip * sj.nprim;
    const double a = exps[si.prim0 + ip], b = exps[sj.prim0 + jp];
    const double* A = geom + 3 * si.atom;
    const double* B = geom + 3 * sj.atom;
    const double p = __dadd_rn(a, b);
    double d2 = 0.0;
    for (int x = 0; x < 3; x++) {
        const double dx = __dadd_rn(A[x], -B[x]);
        d2 = __dadd_rn(d2, __dmul_rn(dx, dx));
        P_p[4 * r + x] = __ddiv_rn(__dadd_rn(__dmul_rn(a, A[x]), __dmul_rn(b, B[x])), p);
        A_a[4 * r + x] = A[x];
        B_b[4 * r + x] = B[x];
    }
    P_p[4 * r + 3] = p;
    A_a[4 * r + 3] = a;
    B_b[4 * r + 3] = b;
    const double gauss = exp(__dmul_rn(__ddiv_rn(__dmul_rn(-a, b), p), d2));
    coef[r] = __dmul_rn(__dmul_rn(coefs[si.prim0 + ip], coefs[sj.prim0 + jp]), gauss);
    i_ao[r] = si.ao;
    j_ao[r] = sj.ao;
    i_atom[r] = si.atom;
    j_atom[r] = sj.atom;
}

// Stream-ordered device buffer: cudaMallocAsync / cudaFreeAsync on the build's
// own stream, so building tables never synchronises the device (other
// streams keep running kernels meanwhile).
template <typename T>
struct DevBuf {
    T* p = nullptr;
    cudaStream_t s = nullptr;
    explicit DevBuf(cudaStream_t stream) : s(stream) {}
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
    cudaError_t alloc(size_t n) { return cudaMallocAsync((void**)&p, sizeof(T) * (n ? n : 1), s); }
};

struct StreamHolder {
    cudaStream_t s = nullptr;
    ~StreamHolder() {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }
};

}  // namespace
}  // namespace eip

using namespace eip;

struct eip_pairs {
    struct Class {
        int n = 0;
        std::vector<double> P, A, B, coef, bound;
        std::vector<int> i_ao, j_ao, i_atom, j_atom;
    };
    std::map<std::pair<int, int>, Class> classes;
    char err[256] = "";
};

namespace {
eip_pairs* pairs_fail(eip_pairs* r, const char* what, cudaError_t e) {
    snprintf(r->err, sizeof r->err, "%s: %s", what, cudaGetErrorString(e));
    fprintf(stderr, "[eip pairs] %s\n", r->err);
    return r;
}
}  // namespace

extern "C" {

eip_pairs* eip_pairs_build(int n_shell, const int* shell_l, const int* shell_atom, const int* shell_ao,
                           const int* shell_nprim, const double* prim_exp, const double* prim_coef, int n_atom,
                           const double* geometry, double threshold) {
    eip_pairs* r = new eip_pairs;
    if (n_shell <= 0 || n_atom <= 0) return r;
    if (int rc = eip_init(-1)) {
        snprintf(r->err, sizeof r->err, "device initialisation failed (%d)", rc);
        return r;
    }
    StreamHolder sth;  // destroyed last: waits for the frees queued below
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&sth.s, cudaStreamNonBlocking)) != cudaSuccess)
        return pairs_fail(r, "stream", e);
    const cudaStream_t st = sth.s;
    std::vector<ShellRec> sh(n_shell);
    int n_prim = 0;
    for (int s = 0; s < n_shell; s++) {
        sh[s] = ShellRec{shell_l[s], shell_atom[s], shell_ao[s], shell_nprim[s], n_prim};
        n_prim += shell_nprim[s];
    }
    DevBuf<ShellRec> d_sh(st);
    DevBuf<double> d_exp(st), d_coef(st), d_geom(st);
    if ((e = d_sh.alloc(n_shell)) || (e = d_exp.alloc(n_prim)) || (e = d_coef.alloc(n_prim)) ||
        (e = d_geom.alloc(3 * (size_t)n_atom)))
        return pairs_fail(r, "allocation", e);
    cudaMemcpyAsync(d_sh.p, sh.data(), sizeof(ShellRec) * n_shell, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_exp.p, prim_exp, sizeof(double) * n_prim, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_coef.p, prim_coef, sizeof(double) * n_prim, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_geom.p, geometry, sizeof(double) * 3 * n_atom, cudaMemcpyHostToDevice, st);
    // shell pairs of each class in the reference's loop order
    std::map<std::pair<int, int>, std::vector<PairRec>> by_class;
    std::map<std::pair<int, int>, int> slots;
    for (int i = 0; i < n_shell; i++)
        for (int j = 0; j < n_shell; j++) {
            if (sh[i].l > sh[j].l || (sh[i].l == sh[j].l && sh[i].ao > sh[j].ao)) continue;
            const std::pair<int, int> key{sh[i].l, sh[j].l};
            int& ns = slots[key];
            by_class[key].push_back(PairRec{i, j, ns});
            ns += sh[i].nprim * sh[j].nprim;
        }
    for (auto& kv : by_class) {
        const int np = (int)kv.second.size(), ns = slots[kv.first];
        DevBuf<PairRec> d_pairs(st);
        DevBuf<double> d_bound(st), d_key(st), d_key_sorted(st);
        DevBuf<int> d_flag(st), d_pos(st), d_val(st), d_val_sorted(st);
        if ((e = d_pairs.alloc(np)) || (e = d_bound.alloc(ns)) || (e = d_flag.alloc(ns)) || (e = d_pos.alloc(ns)) ||
            (e = d_key.alloc(ns)) || (e = d_val.alloc(ns)) || (e = d_key_sorted.alloc(ns)) ||
            (e = d_val_sorted.alloc(ns)))
            return pairs_fail(r, "allocation", e);
        cudaMemcpyAsync(d_pairs.p, kv.second.data(), sizeof(PairRec) * np, cudaMemcpyHostToDevice, st);
        pair_bound_kernel<<<(np + 127) / 128, 128, 0, st>>>(np, d_pairs.p, d_sh.p, d_exp.p, d_coef.p, d_geom.p,
                                                            threshold, d_bound.p);
        flag_kernel<<<(ns + 255) / 256, 256, 0, st>>>(ns, d_bound.p, d_flag.p);
        size_t tmp_bytes = 0, tmp2 = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_flag.p, d_pos.p, ns);
        cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp2, d_key.p, d_key_sorted.p, d_val.p, d_val_sorted.p,
                                                  ns);
        DevBuf<unsigned char> d_tmp(st);
        if ((e = d_tmp.alloc(tmp_bytes > tmp2 ? tmp_bytes : tmp2))) return pairs_fail(r, "allocation", e);
        cub::DeviceScan::ExclusiveSum(d_tmp.p, tmp_bytes, d_flag.p, d_pos.p, ns, st);
        int last[2] = {0, 0};
        cudaMemcpyAsync(&last[0], d_pos.p + ns - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&last[1], d_flag.p + ns - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return pairs_fail(r, "bounds", e);
        const int n_keep = last[0] + last[1];
        if (n_keep == 0) continue;
        compact_kernel<<<(ns + 255) / 256, 256, 0, st>>>(ns, d_bound.p, d_flag.p, d_pos.p, d_key.p, d_val.p);
        // stable: equal bounds keep the insertion (loop) order
        size_t tmp_sort = tmp2;
        cub::DeviceRadixSort::SortPairsDescending(d_tmp.p, tmp_sort, d_key.p, d_key_sorted.p, d_val.p,
                                                  d_val_sorted.p, n_keep, 0, sizeof(double) * 8, st);
        DevBuf<double> P(st), A(st), B(st), coef(st);
        DevBuf<int> iao(st), jao(st), iat(st), jat(st);
        if ((e = P.alloc(4 * (size_t)n_keep)) || (e = A.alloc(4 * (size_t)n_keep)) ||
            (e = B.alloc(4 * (size_t)n_keep)) || (e = coef.alloc(n_keep)) || (e = iao.alloc(n_keep)) ||
            (e = jao.alloc(n_keep)) || (e = iat.alloc(n_keep)) || (e = jat.alloc(n_keep)))
            return pairs_fail(r, "allocation", e);
        pair_rows_kernel<<<(n_keep + 127) / 128, 128, 0, st>>>(n_keep, d_val_sorted.p, np, d_pairs.p, d_sh.p,
                                                               d_exp.p, d_coef.p, d_geom.p, P.p, A.p, B.p, coef.p,
                                                               iao.p, jao.p, iat.p, jat.p);
        if ((e = cudaGetLastError()) != cudaSuccess) return pairs_fail(r, "kernels", e);
        eip_pairs::Class& c = r->classes[kv.first];
        c.n = n_keep;
        c.P.resize(4 * (size_t)n_keep);
        c.A.resize(4 * (size_t)n_keep);
        c.B.resize(4 * (size_t)n_keep);
        c.coef.resize(n_keep);
        c.bound.resize(n_keep);
        c.i_ao.resize(n_keep);
        c.j_ao.resize(n_keep);
        c.i_atom.resize(n_keep);
        c.j_atom.resize(n_keep);
        cudaMemcpyAsync(c.P.data(), P.p, sizeof(double) * 4 * n_keep, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(c.A.data(), A.p, sizeof(double) * 4 * n_keep, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(c.B.data(), B.p, sizeof(double) * 4 * n_keep, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(c.coef.data(), coef.p, sizeof(double) * n_keep, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(c.bound.data(), d_key_sorted.p, sizeof(double) * n_keep, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(c.i_ao.data(), iao.p, sizeof(int) * n_keep, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(c.j_ao.data(), jao.p, sizeof(int) * n_keep, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(c.i_atom.data(), iat.p, sizeof(int) * n_keep, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(c.j_atom.data(), jat.p, sizeof(int) * n_keep, cudaMemcpyDeviceToHost, st);
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
            return pairs_fail(r, "copy", e);
    }
    return r;
}

const char* eip_pairs_error(eip_pairs* r) { return r ? r->err : "null"; }

int eip_pairs_count(eip_pairs* r, int i_L, int j_L) {
    if (!r) return -1;
    auto it = r->classes.find({i_L, j_L});
    return it == r->classes.end() ? 0 : it->second.n;
}

int eip_pairs_copy(eip_pairs* r, int i_L, int j_L, double* P_p, double* A_a, double* B_b, double* coefficient,
                   int* i_ao_start, int* j_ao_start, int* i_atom, int* j_atom, double* upper_bound) {
    if (!r) return 2;
    auto it = r->classes.find({i_L, j_L});
    if (it == r->classes.end()) return 1;
    const eip_pairs::Class& c = it->second;
    memcpy(P_p, c.P.data(), sizeof(double) * c.P.size());
    memcpy(A_a, c.A.data(), sizeof(double) * c.A.size());
    memcpy(B_b, c.B.data(), sizeof(double) * c.B.size());
    memcpy(coefficient, c.coef.data(), sizeof(double) * c.n);
    memcpy(i_ao_start, c.i_ao.data(), sizeof(int) * c.n);
    memcpy(j_ao_start, c.j_ao.data(), sizeof(int) * c.n);
    memcpy(i_atom, c.i_atom.data(), sizeof(int) * c.n);
    memcpy(j_atom, c.j_atom.data(), sizeof(int) * c.n);
    memcpy(upper_bound, c.bound.data(), sizeof(double) * c.n);
    return 0;
}

void eip_pairs_destroy(eip_pairs* r) { delete r; }

}  // extern "C"
