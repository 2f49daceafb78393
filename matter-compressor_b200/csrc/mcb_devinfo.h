// mcb_devinfo.h -- per-device values that the launchers look up once.
//
// A process may drive several GPUs, from several host threads; the values
// (SM count, occupancy, whether a kernel attribute is set) are kept per device
// in atomics. Two threads that race on a first lookup compute and store the
// same value, so no lock is needed.
#pragma once
#include <cuda_runtime.h>

#include <atomic>

namespace mcb {

constexpr int kMaxDevs = 64;

inline int current_device() {
    int dev = 0;
    cudaGetDevice(&dev);
    return dev & (kMaxDevs - 1);
}

// SM count of the current device.
inline int dev_sms() {
    static std::atomic<int> cache[kMaxDevs];
    std::atomic<int> &c = cache[current_device()];
    int v = c.load(std::memory_order_relaxed);
    if (v <= 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        c.store(v, std::memory_order_relaxed);
    }
    return v;
}

// A per-device integer computed once by `f` (called with the device current);
// 0 in the cache means "not computed yet", so `f` must not return 0.
template <class F>
inline int dev_once(std::atomic<int> (&cache)[kMaxDevs], F f) {
    std::atomic<int> &c = cache[current_device()];
    int v = c.load(std::memory_order_acquire);
    if (v == 0) {
        v = f();
        c.store(v, std::memory_order_release);
    }
    return v;
}

}  // namespace mcb
