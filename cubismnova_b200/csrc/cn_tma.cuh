// cn_tma.cuh -- thin inline-PTX wrappers for mbarriers and bulk (TMA) copies.
//
// Only the non-multicast forms are used.  Every wait is bounded: after
// kWaitLimit polls the caller gets `false` and must record an error word.
#pragma once

#include <cstdint>

namespace cn {

constexpr uint32_t kWaitLimit = 1u << 22;

// device error word values
enum : int {
    kDevErrNone = 0,
    kDevErrTimeout = 1,    // an mbarrier wait ran out of polls
    kDevErrBadIndex = 2,   // a table entry pointed outside the grid
    kDevErrBadConfig = 3,  // kernel launched with an unusable configuration
};

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

// make the initialised barrier visible to the async (TMA) proxy
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// 1-D bulk copy global -> shared (TMA engine).  dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gsrc, uint32_t bytes,
                                         uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], "
                 "%2, [%3];" ::"r"(smem_u32(smem_dst)),
                 "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// 5-D tiled TMA load global -> shared (tensor map `tmap`, a generic address
// of a CUtensorMap in parameter, constant or global memory): the map's box
// at coordinates c0..c4 (innermost first, all non-negative, c0 x element
// size a multiple of 16 bytes) lands densely at smem_dst (128-byte aligned);
// completion on `bar`.  No multicast.
__device__ __forceinline__ void tma_load_5d(void *smem_dst, const void *tmap, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                 "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(smem_dst)),
                 "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4),
                 "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}

// Bounded wait; returns false (and leaves the barrier pending) on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        if (mbar_try_wait(bar, parity)) {
            return true;
        }
    }
    return false;
}

// try_wait with a suspend-time hint: while the phase is incomplete the thread
// is suspended for up to `ns` nanoseconds (waking early when the phase
// completes) instead of returning at once, so a whole CTA waiting for a
// bulk copy takes no issue slots from the warps of other CTAs on the SM.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t *bar, uint32_t parity, uint32_t ns)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
                 : "memory");
    return done != 0;
}

constexpr uint32_t kSleepWaitLimit = 1u << 20; // x up to 2 us: about 2 s at most

// Bounded sleeping wait; returns false (barrier left pending) on timeout.
__device__ __forceinline__ bool mbar_wait_bounded_sleep(uint64_t *bar, uint32_t parity, uint32_t ns = 2000)
{
    for (uint32_t i = 0; i < kSleepWaitLimit; ++i) {
        if (mbar_try_wait_sleep(bar, parity, ns)) {
            return true;
        }
    }
    return false;
}

} // namespace cn
