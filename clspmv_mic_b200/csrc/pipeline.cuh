// pipeline.cuh — shared-memory staging with bulk copies (sm_100a): mbarrier
// helpers with bounded waits and the untiled cp.async.bulk global -> shared
// copy, for kernels in which one producer warp streams a format's arrays
// into a ring of stages that consumer warps read.
//
// Every wait is bounded (about 2 s of %globaltimer); a wait that runs out
// adds one to the caller's counter (the kernels pass the device word that
// clspmv_pipeline_timeouts reads) and makes the kernel give up instead of
// spinning for ever.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace clspmv {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void pl_mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// makes the initialised barriers visible to the async proxy (bulk copies)
__device__ __forceinline__ void pl_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ bool pl_mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t pl_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the completion of the barrier's phase with this parity. False
// (and one count in *timeouts) after about 2 s.
__device__ __forceinline__ bool pl_wait(uint32_t bar, uint32_t parity, unsigned int* timeouts)
{
    if (pl_mbar_try(bar, parity)) return true;
    const uint64_t t0 = pl_ns();
    while (!pl_mbar_try(bar, parity)) {
        if (pl_ns() - t0 > 2000000000ull) {
            atomicAdd(timeouts, 1u);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void pl_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// one arrival that also announces `bytes` of bulk copies completing on the barrier
__device__ __forceinline__ void pl_arrive_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// bytes (a multiple of 16; both addresses 16-byte aligned) from global to
// this CTA's shared memory, completing on `bar`
__device__ __forceinline__ void pl_bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar, uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar), "l"(policy)
        : "memory");
}

}  // namespace clspmv
