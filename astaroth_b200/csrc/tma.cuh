// TMA (cp.async.bulk.tensor) and mbarrier primitives for sm_100a, in inline PTX.
//
// Every wait is bounded: a barrier that has not completed after
// ACB_WAIT_LIMIT_NS of wall time makes the wait return false, and the caller
// raises a status bit and leaves instead of spinning forever.
#pragma once
#include <cuda.h>
#include <stdint.h>

#ifndef ACB_WAIT_LIMIT_NS
#define ACB_WAIT_LIMIT_NS 2000000000ull // 2 s
#endif

__device__ __forceinline__ uint32_t
smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void
mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

// Makes barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void
fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void
fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void
mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Plain arrival (no transaction bytes), e.g. a consumer warp releasing a slot.
__device__ __forceinline__ void
mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ uint32_t
mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok;
}

__device__ __forceinline__ uint64_t
global_timer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase with the given parity to complete. Returns false if
// limit_ns of wall time ran out first.
__device__ __forceinline__ bool
mbar_wait_limit(uint64_t* bar, uint32_t parity, uint64_t limit_ns)
{
    if (mbar_try_wait(bar, parity))
        return true;
    const uint64_t t0 = global_timer_ns();
    for (uint32_t it = 0;; ++it) {
        if (mbar_try_wait(bar, parity))
            return true;
        if ((it & 63u) == 63u && global_timer_ns() - t0 > limit_ns)
            return false;
    }
}

// The pipelines' wait: ACB_WAIT_LIMIT_NS.
__device__ __forceinline__ bool
mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    return mbar_wait_limit(bar, parity, ACB_WAIT_LIMIT_NS);
}

// 4-D tiled TMA load (x, y, z, field) into shared memory, completing on `bar`.
// The x coordinate times the element size must be a multiple of 16 bytes;
// the callers guarantee it by construction of the layout and the tiles.
__device__ __forceinline__ void
tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int w, uint64_t* bar)
{
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w),
                 "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void
prefetch_tensormap(const CUtensorMap* map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}
