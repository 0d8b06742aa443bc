// Kernel attributes set once per device.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

namespace kumo_dev {

// Raises a kernel's dynamic shared-memory limit once per device (again only
// for a larger size).  Setting a function attribute while launches of that
// kernel are in flight can hold the calling thread until they end, which a
// serving loop that issues every launch from one thread cannot afford.
inline void ensure_dynamic_smem(const void* func, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    int& have = done[{func, dev}];
    if (have >= bytes) return;
    cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    have = bytes;
}

}  // namespace kumo_dev
