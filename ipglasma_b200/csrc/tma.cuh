// Tensor-memory-accelerator (TMA) copies and shared-memory barriers for
// sm_100a, as inline PTX (PTX ISA: cp.async.bulk.tensor, mbarrier,
// cp.async.bulk.commit_group / wait_group, fence.proxy.async).
//
// Loads complete on an mbarrier with a transaction byte count; stores are
// bulk groups read out of shared memory asynchronously. No load here uses
// cluster multicast: every copy is between this GPU's global memory and the
// issuing CTA's own shared memory. Host side: encode_tiled_3d builds the
// tensor maps through the driver entry point of the runtime (no -lcuda).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace ipg {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

// makes initialised barriers visible to the async proxy (the TMA unit)
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// orders this thread's generic-proxy shared-memory accesses before later
// async-proxy accesses of them (a TMA store reading, a TMA load writing)
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// one arrival that also announces `bytes` of TMA transactions for the phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

// one arrival (release: this thread's earlier shared-memory accesses are
// ordered before the phase completes)
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// waits for the phase of `parity` to complete; false after max_polls polls
// (each try_wait itself suspends for a bounded time)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint32_t max_polls) {
    for (uint32_t i = 0; i < max_polls; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 3-D tiled load of the map's box at (x, y, z) into dst (128-byte aligned);
// completes `bar` with the box's bytes. x * element size must be a multiple
// of 16 bytes; y and z may be negative or past the end (zero fill).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

// 3-D tiled store of src (128-byte aligned) to the map's box at (x, y, z);
// the box must lie inside the tensor (non-negative coordinates)
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, int x, int y, int z,
                                             const void *src) {
    asm volatile(
        "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
            reinterpret_cast<uint64_t>(map)),
        "r"(x), "r"(y), "r"(z), "r"(smem_addr(src))
        : "memory");
}

__device__ __forceinline__ void bulk_commit() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// the shared memory of every committed store has been read
__device__ __forceinline__ void bulk_wait_read_all() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// every committed store has completed
__device__ __forceinline__ void bulk_wait_all() {
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// a tensor map in global memory (written by the host before the launch) is
// acquired by the tensor-map proxy before the first copy through it
__device__ __forceinline__ void fence_map_acquire(const CUtensorMap *map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(
                     reinterpret_cast<uint64_t>(map))
                 : "memory");
}

__device__ __forceinline__ void prefetch_map(const CUtensorMap *map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Host: a 3-D tensor of dims (d0 fastest, d1, d2) of `esize`-byte elements,
// dense, with boxes of (b0, b1, b2), zero fill out of bounds. Returns false
// if the driver rejects it (alignment, strides, box limits).
bool encode_tiled_3d(CUtensorMap *map, void *base, CUtensorMapDataType type, size_t esize,
                     uint64_t d0, uint64_t d1, uint64_t d2, uint32_t b0, uint32_t b1,
                     uint32_t b2);

}  // namespace ipg
