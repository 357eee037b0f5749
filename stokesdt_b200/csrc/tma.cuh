// Tensor-memory-accelerator (TMA) bulk copies and mbarrier waits for the
// grid passes (sm_100a inline PTX).
//
// A pass stages one tile per CTA: thread 0 arms an mbarrier with the tile's
// byte count and issues the tiled bulk load(s); every thread waits on the
// barrier with a bounded number of polls (a timeout sets *err and the CTA
// skips its work instead of spinning forever).  After the transform the tile
// goes back with a tiled bulk store, which reads shared memory asynchronously;
// the issuing thread waits for those reads before the CTA exits.
//
// Rules kept by every caller: the innermost box coordinate times the element
// size is a multiple of 16 bytes; stores never start at a negative
// coordinate; shared-memory tiles are 128-byte aligned.  No copy here uses
// cluster multicast.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace sdt {

// Number of try_wait polls before a wait gives up (each poll may suspend the
// thread for a hardware-defined interval).
constexpr int kMbarPollLimit = 1 << 22;

// Error codes written to the pass error word.
constexpr int kTmaErrTimeout = 1;

// Host: encode a tiled tensor map of 8-byte elements (one float2) of rank
// `rank` (<= 5).  dims[0] is contiguous; strides[i] is the byte stride of
// dimension i+1 (a multiple of 16).  Returns false if the driver entry point
// is missing or rejects the map.
bool encode_tmap_f2(CUtensorMap *map, const void *base, int rank, const unsigned long long *dims,
                    const unsigned long long *strides, const unsigned *box);
// The same for 4-byte (float) or 8-byte elements.
bool encode_tmap(CUtensorMap *map, const void *base, int elem_bytes, int rank,
                 const unsigned long long *dims, const unsigned long long *strides, const unsigned *box);

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

// Make the barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for phase `parity` of the barrier; false after the poll limit.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    for (int i = 0; i < kMbarPollLimit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Tiled bulk load of a 3D / 4D box into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0,
                                            int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0,
                                            int c1, int c2, int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2),
        "r"(c3)
        : "memory");
}

// Tiled bulk stores from shared memory (bulk-group completion).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int c0, int c1,
                                             int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
            reinterpret_cast<uint64_t>(map)),
        "r"(smem_addr(src)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

__device__ __forceinline__ void tma_store_4d(const CUtensorMap *map, const void *src, int c0, int c1,
                                             int c2, int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5}], [%1];" ::"l"(
            reinterpret_cast<uint64_t>(map)),
        "r"(smem_addr(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}

// Untiled bulk load of `bytes` (a multiple of 16; both addresses 16-byte
// aligned) into shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// Wait until the committed bulk stores have finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read_all()
{
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Order this thread's generic-proxy shared-memory writes before later
// async-proxy (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace sdt
