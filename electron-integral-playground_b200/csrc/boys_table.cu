// Device-resident constant tables: the Boys-function Taylor grid and run-time
// copies of the spherical-harmonic / normalisation coefficients.
#include <math.h>

#include <mutex>

#include "eip_common.cuh"
#include "eip_internal.h"

namespace eip {

// order-major: row (L, i) = F_L..F_{L+kBoysTaylor-1}(T0_i), 64-byte aligned (boys_row)
constexpr size_t kBoysTableDoubles = (size_t)(kMaxBoysM + 1) * kBoysGrid * kBoysTaylor;
__device__ __align__(64) double g_boys_table[kBoysTableDoubles];

namespace {
// Device address of g_boys_table per device (nullptr: tables not uploaded yet).
std::atomic<const double*> g_boys_address[kMaxDevices];
std::mutex g_tables_mu;
}  // namespace

// F_m(T0) on the grid: F_M(T0) = e^-T0 sum_k (2 T0)^k / ((2M+1)(2M+3)...(2M+2k+1))
// (all terms positive: no cancellation), in long double, then the downward
// recursion F_m = (2 T0 F_{m+1} + e^-T0) / (2m+1) for the lower orders.
static void build_boys_table(double* out) {
    const int M = kBoysOrders - 1;
    for (int i = 0; i < kBoysGrid; i++) {
        long double T = (long double)i * (long double)kBoysStep;
        long double eT = expl(-T);
        long double F[kBoysOrders];
        long double term = 1.0L / (2 * M + 1), sum = term;
        for (int k = 1; k < 10000; k++) {
            term *= 2.0L * T / (2 * M + 2 * k + 1);
            sum += term;
            if (term < sum * 1e-22L) break;
        }
        F[M] = eT * sum;
        for (int m = M - 1; m >= 0; m--) F[m] = (2.0L * T * F[m + 1] + eT) / (2 * m + 1);
        for (int L = 0; L <= kMaxBoysM; L++)
            for (int k = 0; k < kBoysTaylor; k++)
                out[((size_t)L * kBoysGrid + i) * kBoysTaylor + k] = (double)F[L + k];
    }
}

int ensure_device_tables() {
    const int dev = current_device();
    if (dev < 0) return (int)cudaErrorInvalidDevice;
    if (g_boys_address[dev].load(std::memory_order_acquire)) return 0;
    std::lock_guard<std::mutex> lock(g_tables_mu);
    if (g_boys_address[dev].load(std::memory_order_acquire)) return 0;
    static double host_table[kBoysTableDoubles];
    static bool built = false;
    if (!built) {
        build_boys_table(host_table);
        built = true;
    }
    cudaError_t e = cudaMemcpyToSymbol(g_boys_table, host_table, sizeof(host_table));
    void* addr = nullptr;
    if (e == cudaSuccess) e = cudaGetSymbolAddress(&addr, g_boys_table);
    if (e != cudaSuccess) return (int)e;
    if (int rc = upload_generic_tables()) return rc;
    // published last: a non-null address means every table of the device is in place
    g_boys_address[dev].store(static_cast<const double*>(addr), std::memory_order_release);
    return 0;
}

const double* boys_table_device() {
    const int dev = current_device();
    if (dev < 0) return nullptr;
    const double* t = g_boys_address[dev].load(std::memory_order_acquire);
    if (t) return t;
    return ensure_device_tables() == 0 ? g_boys_address[dev].load(std::memory_order_acquire) : nullptr;
}

// Evaluate F_0..F_L on the device for a list of T (tests the device Boys).
__global__ void boys_probe_kernel(const double* __restrict__ table, int L, const double* T, int n, double* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double F[kMaxBoysM + 1];
    boys_rt(table, L, T[i], F);
    for (int m = 0; m <= L; m++) out[(size_t)i * (L + 1) + m] = F[m];
}

int launch_boys_probe(int L, const double* dT, int n, double* dout, cudaStream_t s) {
    if (L < 0 || L > kMaxBoysM) return 1;
    if (n <= 0) return 0;
    const double* table = boys_table_device();
    if (!table) return 2;
    boys_probe_kernel<<<(n + 127) / 128, 128, 0, s>>>(table, L, dT, n, dout);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace eip
