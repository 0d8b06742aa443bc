// Kernel attributes set once per device.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>
#include <vector>

namespace kumo_dev {

// Every kernel instantiation the library launches, listed while the library
// loads: a launch site names its kernel with KUMO_REGISTER_KERNEL, whose
// class-template static member adds the kernel to the list during static
// initialisation, before any launch.  preload_kernels() asks CUDA for each
// listed kernel's attributes once per device, which loads it; otherwise CUDA
// loads a kernel at its first launch, and every host thread launching
// meanwhile waits.  Defined in csrc/host/evaluator.cu.
std::vector<const void*>& kernel_registry();
void preload_kernels();

inline bool register_kernel(const void* func) {
    kernel_registry().push_back(func);
    return true;
}

template <auto Func>
struct KernelEntry {
    static inline const bool registered = register_kernel(reinterpret_cast<const void*>(Func));
};

#define KUMO_REGISTER_KERNEL(...) (void)::kumo_dev::KernelEntry<&__VA_ARGS__>::registered

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
