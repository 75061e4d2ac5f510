// ysg_tma.cuh -- bulk (TMA) copy of the model table into shared memory.
//
// One elected thread arms an mbarrier with the byte count and issues
// cp.async.bulk global->shared copies; every thread then waits on the
// barrier phase.  The wait is bounded: after ~1 s of polling the kernel sets
// a status bit, waits once more (also bounded) for the copy in flight and
// reports failure so the caller can return instead of hanging.  No
// multicast is used; the source is always this GPU's own memory.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ysg {

constexpr int STATUS_TMA_TIMEOUT = 1;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count)
                 : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(mbar))
        : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* mbar, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(mbar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Poll the barrier for at most ~max_iter * 128 ns.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* mbar, uint32_t phase, int max_iter)
{
    for (int it = 0; it < max_iter; it++) {
        if (mbar_test(mbar, phase)) return true;
        __nanosleep(128);
    }
    return false;
}

// Copy `bytes` (a multiple of 16; both addresses 16-byte aligned) from
// global to shared memory.  Must be called by every thread of the block.
// Returns false (and sets STATUS_TMA_TIMEOUT in *status) if the copy did not
// complete within the bounded wait.
__device__ inline bool stage_to_smem(void* dst, const void* src, uint32_t bytes, uint64_t* mbar,
                                     int* status)
{
    if (threadIdx.x == 0) {
        mbar_init(mbar, 1);
        mbar_expect_tx(mbar, bytes);
        const uint32_t chunk = 32768;
        for (uint32_t off = 0; off < bytes; off += chunk) {
            uint32_t n = bytes - off < chunk ? bytes - off : chunk;
            bulk_g2s((char*)dst + off, (const char*)src + off, n, mbar);
        }
    }
    __syncthreads();
    bool ok = mbar_wait_bounded(mbar, 0, 1 << 23);
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(status, STATUS_TMA_TIMEOUT);
        mbar_wait_bounded(mbar, 0, 1 << 20);
    }
    // every thread must agree before any leaves
    return __syncthreads_and(ok ? 1 : 0) != 0;
}

}  // namespace ysg
