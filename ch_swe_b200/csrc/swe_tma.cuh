// swe_tma.cuh -- tensor-memory-accelerator (TMA) tile loads into shared memory and
// the mbarrier they complete on, for the fused stage kernels (sm_100a).
//
// One elected thread arms an mbarrier with the byte count of a batch of 2-D tile
// loads and issues them; every thread then waits on the barrier's phase.  The
// waits are bounded (a second of global time): a wait that runs out reports
// failure to the caller, which records an error flag and leaves the kernel
// instead of spinning for ever.  No load here uses cluster multicast: every
// tensor map covers this GPU's own memory.
#pragma once

#include <cuda.h>   // CUtensorMap

#include <cstdint>

namespace chswe {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make an initialised barrier (and shared memory written by threads) visible to
// the asynchronous proxy that the tile loads run in.
__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `parity` of the barrier for at most limit_ns nanoseconds (the clock is
// read every 256 polls).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns)
{
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1;; it++) {
        if (mbar_test(bar, parity)) return true;
        if ((it & 255u) == 0 && global_ns() - t0 > limit_ns) return false;
    }
}

// One 2-D tile of a tensor map into shared memory at dst (128-byte aligned),
// completing `box bytes` of transactions on bar.  x (innermost, in elements) times
// the element size must be a multiple of 16 bytes; coordinates past the tensor's
// extent read zeros.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)map) : "memory");
}

// Loads through L2 only: data another kernel of the same stage chain wrote.
template <class T>
__device__ __forceinline__ T ld_cg(const T *p)
{
    return __ldcg(p);
}

}  // namespace chswe
