// Tensor Memory Accelerator helpers for sm_100a: mbarrier, 2D tiled and 1D bulk copies global -> shared memory.
// Every wait is bounded: after TMA_WAIT_LIMIT polls the caller gives up and reports W2B_ETIMEOUT. Every copy here
// lands in the shared memory of the one CTA that issues it, from this GPU's own memory.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace w2b {

constexpr uint32_t TMA_WAIT_LIMIT = 1u << 18;  // about 1 s: a poll that finds the phase open takes about 4 us

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make the barrier's initialisation visible to the asynchronous proxy (the TMA unit).
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Order this thread's earlier generic-proxy accesses of shared memory before later async-proxy ones (a TMA write
// into a buffer the CTA has just read).
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Wait for the barrier's phase; false if the wait gave up (after `limit` polls: TMA_WAIT_LIMIT everywhere but in the
// wait's own self-check).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, uint32_t limit = TMA_WAIT_LIMIT) {
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

// A 2D box of a tensor map into shared memory; x is the innermost coordinate (its byte offset is a multiple of 16).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// A contiguous run of bytes (16-byte aligned, a multiple of 16 long) into shared memory.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

}  // namespace w2b
