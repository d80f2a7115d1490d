// Per-device cache of the dynamic shared-memory attribute of a kernel.
#pragma once
#include <cuda_runtime.h>

#include <atomic>

namespace flb {

// cudaFuncSetAttribute(max dynamic shared memory) once per kernel and device:
// the attribute belongs to the device's context, so a process that solves on
// several GPUs sets it on each (one bit per device in `devs`)
template <typename K>
inline cudaError_t smem_attr_once(std::atomic<unsigned long long>& devs, K kernel, size_t smem) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (devs.load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) devs.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

}  // namespace flb
