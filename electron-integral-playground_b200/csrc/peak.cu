// FMA-throughput microbenchmark: the FP64 / FP32 roofline denominators of the
// integral kernels (the measured-peaks file of the box has HBM and bf16 only).
// Eight independent FMA chains per thread; grid of 8 CTAs x 256 threads per SM.
#include <cuda_runtime.h>

#include "../../include/eip_b200.h"

namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_chains(T* out, int iters, T a, T b) {
    T x0 = threadIdx.x * (T)1e-3, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
    T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == (T)-12345.0) out[blockIdx.x] = s;  // keeps the chains live
}

template <typename T>
int measure(double* tflops) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 2;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    T* out = nullptr;
    if (cudaMalloc(&out, sizeof(T) * 8 * sms) != cudaSuccess) return 2;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = 8 * sms, threads = 256, iters = sizeof(T) == 8 ? 2048 : 4096;
    fma_chains<T><<<blocks, threads>>>(out, 64, (T)0.999999, (T)1e-7);  // warm-up
    double best = 0.0;
    for (int r = 0; r < 5; r++) {
        cudaEventRecord(e0);
        fma_chains<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 64.0 * iters * (double)blocks * threads;
        if (ms > 0) best = flops / (ms * 1e-3) / 1e12 > best ? flops / (ms * 1e-3) / 1e12 : best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *tflops = best;
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace

extern "C" int eip_measure_fma_peak(int fp64, double* tflops) {
    return fp64 ? measure<double>(tflops) : measure<float>(tflops);
}
