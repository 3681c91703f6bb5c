// Per-device state of the library: which device a call runs on, the constant
// tables each device holds, and the launch attributes set per device.
//
// Module data (the Boys grid, the constant-memory coefficient tables) and
// function attributes exist once per device, so each is set up the first time
// the library is used with that device current, under a lock, and looked up
// by the current device at every launch.  A process may use several devices
// (one after the other or from several host threads).
#include <mutex>

#include "eip_common.cuh"
#include "eip_internal.h"

namespace eip {

int current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -1;
    return dev;
}

namespace {
std::mutex g_attr_mu;
}

int persistent_grid(const void* kernel, int threads, size_t smem_bytes, std::atomic<int>* cache) {
    const int dev = current_device();
    if (dev < 0) return 0;
    int v = cache[dev].load(std::memory_order_acquire);
    if (v > 0) return v;
    std::lock_guard<std::mutex> lock(g_attr_mu);
    v = cache[dev].load(std::memory_order_acquire);
    if (v > 0) return v;
    int per_sm = 0, sms = 0;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes) != cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem_bytes) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    v = (per_sm < 1 ? 1 : per_sm) * sms;
    cache[dev].store(v, std::memory_order_release);
    return v;
}

}  // namespace eip
