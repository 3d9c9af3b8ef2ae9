// team_sync.cuh -- mbarrier and bulk-copy helpers of the team kernels (inline PTX for sm_100a).
//
// Every wait is bounded: mbar_wait gives up after a number of polls and returns false.  The team kernels
// then wait (bounded again) for their copies in flight, set bit 0 of their error word and end the CTA, so a
// copy that never completes ends the launch with an error status that the host reads, not a hung GPU.
#pragma once
#include <cstdint>

namespace qcg {
namespace team {

// a wait for a bulk copy gives up after this many polls (each poll may suspend the thread for a while)
constexpr long long kWaitPolls = 1ll << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from global to shared memory,
// completing a phase of `bar`
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// bounded wait for phase `parity` of `bar`; false when it gave up after `polls` polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long polls = kWaitPolls)
{
    for (long long n = 0; n < polls; ++n)
    {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// After the wait for step `step` of a stream of `nsteps` stages (stage of step x: base + x, three deep, the
// copy of step x issued while step x - 2 is consumed) gave up: wait, bounded, for the copies still in
// flight -- steps `step` and `step` + 1 -- so that none lands in this CTA's shared memory after it exited.
__device__ __forceinline__ void drain(uint64_t* full, unsigned long long base, int step, int nsteps)
{
    for (int x = step; x < nsteps && x <= step + 1; ++x)
    {
        const unsigned long long gs = base + x;
        mbar_wait(&full[gs % 3], (uint32_t)((gs / 3) & 1));
    }
}

// the barrier's memory may be reused for other data afterwards
__device__ __forceinline__ void mbar_inval(uint64_t* bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// this thread's generic-proxy writes to global memory become visible to later bulk copies (async proxy)
__device__ __forceinline__ void fence_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

}   // namespace team

}   // namespace qcg
