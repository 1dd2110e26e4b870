// tma.cuh — tensor-memory-accelerator (TMA) staging of 2-D boxes into shared memory.
//
// One thread arms an mbarrier with the bytes it expects and issues cp.async.bulk.tensor loads of
// tiled boxes described by CUtensorMaps (built on the host by cuTensorMapEncodeTiled); the copy
// engine writes the boxes into shared memory and completes the transaction on the barrier, and
// every thread waits on the barrier's phase. Loads read this GPU's own memory only and never use
// cluster multicast.
//
// Rules the callers keep: a box's innermost coordinate times the element size is a multiple of
// 16 bytes; its shared-memory destination is 128-byte aligned; the barrier is initialised once
// per CTA and every wait is bounded (on time-out the caller records an error and goes on).
#pragma once

#include <cuda.h>
#include <cstdint>

namespace wcb {

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the copy engine (the async proxy)
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// A tiled 2-D box at (x, y) of `map` into shared memory at dst; completes on `bar`.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// Waits for phase `parity` of `bar` for at most `limit_ns`; false if it timed out.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned long long limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    unsigned long long t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > limit_ns) return false;
    }
}

}  // namespace wcb
