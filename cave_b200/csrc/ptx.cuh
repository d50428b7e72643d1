// ptx.cuh -- inline-PTX helpers for mbarriers and TMA bulk copies (sm_90+ forms used on sm_100a).
// Only non-multicast bulk copies are used anywhere in this library.
#pragma once
#include "cave_stdint.h"

namespace cave {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Dynamic shared memory of the launch, in bytes.
__device__ __forceinline__ uint32_t dynamic_smem_bytes() {
    uint32_t r;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(r));
    return r;
}
// Warp-wide reductions (redux.sync, one instruction each) over all 32 lanes; every lane gets
// the result. volatile: they must stay where all 32 lanes execute them.
__device__ __forceinline__ uint32_t warp_add(uint32_t v) {
    uint32_t r;
    asm volatile("redux.sync.add.u32 %0, %1, 0xffffffff;" : "=r"(r) : "r"(v));
    return r;
}
__device__ __forceinline__ uint32_t warp_min(uint32_t v) {
    uint32_t r;
    asm volatile("redux.sync.min.u32 %0, %1, 0xffffffff;" : "=r"(r) : "r"(v));
    return r;
}
__device__ __forceinline__ uint32_t warp_max(uint32_t v) {
    uint32_t r;
    asm volatile("redux.sync.max.u32 %0, %1, 0xffffffff;" : "=r"(r) : "r"(v));
    return r;
}
__device__ __forceinline__ uint32_t warp_or(uint32_t v) {
    uint32_t r;
    asm volatile("redux.sync.or.b32 %0, %1, 0xffffffff;" : "=r"(r) : "r"(v));
    return r;
}
// One tick's per-thread statistics v[0..10) reduced over the warp: 0..3 sums, 4..6 minima,
// 7..9 maxima (the bounding box).
__device__ __forceinline__ void warp_reduce_tick(uint32_t* v) {
#pragma unroll
    for (int q = 0; q < 4; q++) v[q] = warp_add(v[q]);
#pragma unroll
    for (int q = 4; q < 7; q++) v[q] = warp_min(v[q]);
#pragma unroll
    for (int q = 7; q < 10; q++) v[q] = warp_max(v[q]);
}
// Nanoseconds of the GPU's global timer.
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits for phase `parity` of `bar`, giving up after `limit_ns` nanoseconds (returns false
// then). The first poll needs no timer read.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (global_ns() - t0 > limit_ns) return false;
    }
    return true;
}
// Bulk global->shared copy (no multicast), completion signalled on `bar`. dst, src and bytes
// must be multiples of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// Orders this thread's generic-proxy shared-memory accesses before later async-proxy ones.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace cave
