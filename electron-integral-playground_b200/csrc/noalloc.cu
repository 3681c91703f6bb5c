// eip_three_center_noalloc: (mu nu|P) of one angular class with every buffer
// on the device and no memory allocated by the library.
//
// Some callers cannot let a library call cudaMalloc: code that runs while the
// device memory is owned by another allocator (a framework's caching pool, a
// host program that reserves all device memory up front), code on a path where
// an allocation could block or fail at an unpredictable time (a real-time
// loop, a process near its memory limit), and code that must not synchronise
// the device, which cudaMalloc / cudaFree may do.  For them this entry point
// computes the same integrals as three_center() but takes device pointers and a
// stream, and keeps its working memory in one fixed file-scope device array.
//
// Working memory: g_noalloc_scratch, kNoAllocScratchBytes = 16 MiB, allocated
// with the module on every GPU that loads the library and held until the
// process exits.  A call needs, for its n_pair x n_aux_primitive primitive
// triplets, the converted input tables, a one-molecule work list and one
// output block per primitive triplet; a call that needs more is rejected with
// status 4 (eip_last_error() says why), before anything is launched.
//
// Every call on the device shares that array, and the array keeps the last
// call's contents.  The only words that must start at zero, the work counter
// and status of the integral kernel, are cleared by the call's first kernel;
// every other word a call reads it has written itself.  Two calls whose kernels overlap on the GPU (different
// streams, or different host threads, without ordering) race on the array:
// callers must order them, e.g. issue all calls on one stream.
//
// Set-up: the first call on each device (with that device current) looks up
// the array's device address with cudaGetSymbolAddress and uploads the
// library's constant tables (Boys grid, spherical coefficients) with
// cudaMemcpyToSymbol, once per device under a lock (several host threads may
// make first calls at once); make that first call before any stream capture.
// Later calls only launch kernels on the given stream, asynchronously.
//
// eip_three_center_noalloc_check() computes a call's working-memory need on
// the host (no CUDA call), so a caller can split its work before calling.
#include <stdio.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "eip_common.cuh"
#include "eip_internal.h"
#include "../../include/eip_b200.h"

namespace eip {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr int kNoAllocMaxAuxPrimitives = 65535;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device; null until that device's set-up.
std::atomic<unsigned char*> g_scratch_address[kMaxDevices];
std::mutex g_setup_mu;

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Byte offsets of one call's arrays in the scratch array.
struct ScratchLayout {
    size_t bbeg, bao, bab, bp, bpa, kbeg, kst, kc, kco, misc, pk, total;
};

ScratchLayout scratch_layout(int i_L, int j_L, int k_L, size_t np, size_t na, bool spherical) {
    const size_t ni = spherical ? nsph(i_L) : ncart(i_L), nj = spherical ? nsph(j_L) : ncart(j_L),
                 nk = spherical ? nsph(k_L) : ncart(k_L);
    ScratchLayout l{};
    size_t off = 0;
    l.bbeg = off; off += align256(sizeof(int) * (np + 1));
    l.bao = off; off += align256(sizeof(int2) * np);
    l.bab = off; off += align256(sizeof(double4) * np);
    l.bp = off; off += align256(sizeof(double4) * np);
    l.bpa = off; off += align256(sizeof(double4) * np);
    l.kbeg = off; off += align256(sizeof(int) * (na + 1));
    l.kst = off; off += align256(sizeof(int) * na);
    l.kc = off; off += align256(sizeof(double4) * na);
    l.kco = off; off += align256(sizeof(double) * na);
    l.misc = off; off += align256(16 * sizeof(int) + sizeof(long long));
    l.pk = off; off += align256(sizeof(double) * np * na * ni * nj * nk);
    l.total = off;
    return l;
}

bool class_supported(int i_L, int j_L, int k_L) {
    return i_L >= 0 && j_L >= 0 && k_L >= 0 && i_L <= j_L && j_L <= kMaxOrbitalL && k_L <= kMaxAuxL;
}

// Device address of the scratch array on the current device, setting the
// device up (address lookup, constant tables) on its first call; null on failure.
unsigned char* scratch_on_current_device() {
    const int dev = current_device();
    if (dev < 0) {
        set_error("eip_three_center_noalloc: no usable CUDA device", cudaGetLastError());
        return nullptr;
    }
    unsigned char* p = g_scratch_address[dev].load(std::memory_order_acquire);
    if (p) return p;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    p = g_scratch_address[dev].load(std::memory_order_acquire);
    if (p) return p;
    void* addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess || addr == nullptr) {
        set_error("eip_three_center_noalloc: cudaGetSymbolAddress", e);
        return nullptr;
    }
    if (int rc = ensure_device_tables()) {
        set_error("eip_three_center_noalloc: constant table upload", (cudaError_t)rc);
        return nullptr;
    }
    p = static_cast<unsigned char*>(addr);
    g_scratch_address[dev].store(p, std::memory_order_release);
    return p;
}

// Reference-format device arrays -> the general kernel's tables, one group per
// primitive pair and per auxiliary primitive (no grouping: nothing to sort),
// and its one-molecule work list: misc[0..3] counter and status (cleared),
// [4..5] item begin, [6..7] pair begin, [8..9] auxiliary begin; out_begin = 0.
__global__ void noalloc_tables_kernel(const double* __restrict__ P_p, const double* __restrict__ A_a,
                                      const double* __restrict__ B_b, const double* __restrict__ coef,
                                      const int* __restrict__ ia, const int* __restrict__ ja, int n_pair,
                                      const double* __restrict__ C_q, const double* __restrict__ aux_coef,
                                      const int* __restrict__ aux_start, int n_aux, int* bra_begin, int2* bra_ao,
                                      double4* bra_AB, double4* bra_P, double4* bra_PA, int* ket_begin,
                                      int* ket_start, double4* ket_C, double* ket_coef, int* misc,
                                      long long* out_begin, int items) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        const int m[10] = {0, 0, 0, 0, 0, items, 0, n_pair, 0, n_aux};
        for (int k = 0; k < 10; k++) misc[k] = m[k];
        *out_begin = 0;
    }
    if (i <= n_pair) bra_begin[i] = i;
    if (i <= n_aux) ket_begin[i] = i;
    if (i < n_pair) {
        const double* P = P_p + 4 * (size_t)i;
        const double* A = A_a + 4 * (size_t)i;
        const double* B = B_b + 4 * (size_t)i;
        bra_ao[i] = make_int2(ia[i], ja[i]);
        bra_AB[i] = make_double4(A[0] - B[0], A[1] - B[1], A[2] - B[2], 0.0);
        bra_P[i] = make_double4(P[0], P[1], P[2], P[3]);
        bra_PA[i] = make_double4(P[0] - A[0], P[1] - A[1], P[2] - A[2], coef[i]);
    }
    if (i < n_aux) {
        const double* C = C_q + 4 * (size_t)i;
        ket_start[i] = aux_start[i];
        ket_C[i] = make_double4(C[0], C[1], C[2], C[3]);
        ket_coef[i] = aux_coef[i];
    }
}

// packed[((pair * ni + I) * nj + J) * nk + K) * n_aux + a] -> J3c += (mirrored like
// MI/three_center.cpp:242-244); primitive pairs of one shell pair add into
// the same elements, hence the atomics.
__global__ void noalloc_scatter_kernel(const double* __restrict__ packed, const int2* __restrict__ bra_ao,
                                       const int* __restrict__ ket_start, int n_pair, int n_aux, int ni, int nj,
                                       int nk, double* J3c, int n_ao) {
    const long long total = (long long)n_pair * ni * nj * nk * n_aux;
    const size_t nao = (size_t)n_ao;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long r = e;
        const int a = (int)(r % n_aux); r /= n_aux;
        const int K = (int)(r % nk); r /= nk;
        const int J = (int)(r % nj); r /= nj;
        const int I = (int)(r % ni); r /= ni;
        const int p = (int)r;
        const int2 ao = bra_ao[p];
        const size_t k0 = (size_t)ket_start[a] + K;
        const double v = packed[e];
        atomicAdd(J3c + k0 * nao * nao + (size_t)(ao.x + I) * nao + (ao.y + J), v);
        if (ao.x != ao.y) atomicAdd(J3c + k0 * nao * nao + (size_t)(ao.y + J) * nao + (ao.x + I), v);
    }
}

}  // namespace
}  // namespace eip

using namespace eip;

extern "C" size_t eip_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

extern "C" int eip_three_center_noalloc_check(const int i_L, const int j_L, const int k_L, const int n_pair_ij,
                                              const int n_aux_primitive_k, const bool spherical,
                                              size_t* bytes_needed) {
    if (bytes_needed) *bytes_needed = 0;
    if (!class_supported(i_L, j_L, k_L)) return 1;
    if (n_pair_ij <= 0 || n_aux_primitive_k <= 0) return 0;
    const ScratchLayout l = scratch_layout(i_L, j_L, k_L, (size_t)n_pair_ij, (size_t)n_aux_primitive_k, spherical);
    if (bytes_needed) *bytes_needed = l.total;
    return l.total > kNoAllocScratchBytes || n_aux_primitive_k > kNoAllocMaxAuxPrimitives ? 4 : 0;
}

extern "C" int eip_three_center_noalloc(const int i_L, const int j_L, const int k_L, const double* pair_P_p,
                                        const double* pair_A_a, const double* pair_B_b,
                                        const double* pair_coefficient, const int* pair_i_ao_start,
                                        const int* pair_j_ao_start, const int n_pair_ij, const double* aux_A_a,
                                        const double* aux_coefficient, const int* aux_i_aux_start,
                                        const int n_aux_primitive_k, double* J3c_matrix, const int n_ao,
                                        const int n_aux, const bool spherical, const double omega, void* stream) {
    (void)n_aux;
    size_t need = 0;
    const int fit = eip_three_center_noalloc_check(i_L, j_L, k_L, n_pair_ij, n_aux_primitive_k, spherical, &need);
    if (fit == 1) {
        printf("%s function does not support angular i_L = %d, j_L = %d, k_L = %d\n", __func__, i_L, j_L, k_L);
        fflush(stdout);
        return 1;
    }
    if (n_pair_ij <= 0 || n_aux_primitive_k <= 0) return 0;
    if (fit == 4) {
        char msg[384];
        snprintf(msg, sizeof msg,
                 "eip_three_center_noalloc: class (%d%d|%d) with %d primitive pairs x %d auxiliary primitives needs "
                 "%zu bytes of working memory; the fixed limit is %zu bytes and %d auxiliary primitives: split the "
                 "call or use three_center()",
                 i_L, j_L, k_L, n_pair_ij, n_aux_primitive_k, need, kNoAllocScratchBytes, kNoAllocMaxAuxPrimitives);
        set_error(msg, cudaSuccess);
        return 4;
    }
    unsigned char* s = scratch_on_current_device();
    if (!s) return 2;
    const size_t np = (size_t)n_pair_ij, na = (size_t)n_aux_primitive_k;
    const int ni = spherical ? nsph(i_L) : ncart(i_L), nj = spherical ? nsph(j_L) : ncart(j_L),
              nk = spherical ? nsph(k_L) : ncart(k_L);
    const ScratchLayout l = scratch_layout(i_L, j_L, k_L, np, na, spherical);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nmax = (int)std::max(np, na) + 1;
    const long long items = (long long)np * na * general_chunks(i_L, j_L, k_L, false, spherical);
    int* misc = reinterpret_cast<int*>(s + l.misc);
    long long* out_begin = reinterpret_cast<long long*>(s + l.misc + 16 * sizeof(int));
    noalloc_tables_kernel<<<(nmax + 127) / 128, 128, 0, st>>>(
        pair_P_p, pair_A_a, pair_B_b, pair_coefficient, pair_i_ao_start, pair_j_ao_start, n_pair_ij, aux_A_a,
        aux_coefficient, aux_i_aux_start, n_aux_primitive_k, reinterpret_cast<int*>(s + l.bbeg),
        reinterpret_cast<int2*>(s + l.bao), reinterpret_cast<double4*>(s + l.bab),
        reinterpret_cast<double4*>(s + l.bp), reinterpret_cast<double4*>(s + l.bpa),
        reinterpret_cast<int*>(s + l.kbeg), reinterpret_cast<int*>(s + l.kst), reinterpret_cast<double4*>(s + l.kc),
        reinterpret_cast<double*>(s + l.kco), misc, out_begin, (int)items);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("eip_three_center_noalloc: table kernel launch", e);
        return 2;
    }
    BraTable bra{n_pair_ij, reinterpret_cast<int*>(s + l.bbeg), reinterpret_cast<int2*>(s + l.bao),
                 reinterpret_cast<double4*>(s + l.bab), reinterpret_cast<double4*>(s + l.bp),
                 reinterpret_cast<double4*>(s + l.bpa), nullptr};
    KetTable ket{n_aux_primitive_k, reinterpret_cast<int*>(s + l.kbeg), reinterpret_cast<int*>(s + l.kst),
                 reinterpret_cast<double4*>(s + l.kc), reinterpret_cast<double*>(s + l.kco)};
    double* packed = reinterpret_cast<double*>(s + l.pk);
    BatchMap map{1, misc + 4, misc + 6, misc + 8, out_begin, nullptr, nullptr, nullptr};
    int rc = launch_general(i_L, j_L, k_L, false, spherical, bra, ket, map, (int)items, omega, packed, misc, st);
    if (rc == 0) {
        const long long total = (long long)np * ni * nj * nk * na;
        long long blocks = (total + 255) / 256;
        if (blocks > 148 * 32) blocks = 148 * 32;
        noalloc_scatter_kernel<<<(unsigned)blocks, 256, 0, st>>>(packed, bra.grp_ao, ket.grp_start, n_pair_ij,
                                                                  n_aux_primitive_k, ni, nj, nk, J3c_matrix, n_ao);
        rc = cudaGetLastError() == cudaSuccess ? 0 : 2;
    }
    if (rc != 0) {
        set_error("eip_three_center_noalloc: kernel launch", cudaGetLastError());
        return 2;
    }
    return 0;
}
