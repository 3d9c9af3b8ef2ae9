// smem_attr.h -- the dynamic shared-memory limit above 48 KB is an attribute of a kernel on ONE device.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>

namespace qcg {

// Set it once per (kernel, device), remembered in a bit mask per call site (devices 0..63), so that every
// GPU of the process gets it.  Two threads setting it at once is harmless.
template <class KernelPtr>
inline void ensure_smem(KernelPtr k, size_t smem, std::atomic<unsigned long long>& ready)
{
    if (smem <= 48 * 1024) return;
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (ready.load(std::memory_order_acquire) & bit) return;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    ready.fetch_or(bit, std::memory_order_release);
}

}   // namespace qcg
