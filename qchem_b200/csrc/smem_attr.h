// smem_attr.h -- the dynamic shared-memory limit above 48 KB is an attribute of a kernel on ONE device.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>

namespace qcg {

// Set it once per (kernel, device), remembered in a bit mask per call site (devices 0..63), so that every
// GPU of the process gets it.  It is set for any dynamic size: the default 48 KB limit covers the kernel's
// static shared memory too, so a dynamic size just under 48 KB can already need it.  Two threads setting
// it at once is harmless.
template <class KernelPtr>
inline void ensure_smem(KernelPtr k, size_t smem, std::atomic<unsigned long long>& ready)
{
    if (smem == 0) return;
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (ready.load(std::memory_order_acquire) & bit) return;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    ready.fetch_or(bit, std::memory_order_release);
}

}   // namespace qcg
