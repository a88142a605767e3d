// tma.cuh -- Tensor Memory Accelerator helpers for sm_100a: mbarrier
// synchronisation and 4-D tiled bulk tensor loads (cp.async.bulk.tensor) into
// shared memory, written as inline PTX from the PTX ISA; plus the host-side
// tensor-map encoder (cuTensorMapEncodeTiled through the runtime's driver
// entry point, so libcuda is not linked directly).
//
// Alignment contract (checked by every caller before a copy is issued): the
// innermost coordinate times 8 bytes is a multiple of 16 (even for doubles),
// shared destinations are 128-byte aligned, every mbarrier wait is bounded.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace how {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// 4-byte asynchronous global -> shared copy (both addresses 4-byte aligned)
// and its group commit / wait
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// all but the most recent commit group of this thread have landed
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// make mbarrier initialisation visible to the async (TMA) proxy
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order this thread's earlier generic-proxy shared accesses before later
// async-proxy (TMA) writes to the same shared memory
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase: gives up after `limit` polls and returns
// false (the caller records an error status; nothing spins forever).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 4-D tiled tensor load global -> shared, completion counted on `bar`.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2, int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}

// Host: encode a 4-D FP64 tensor map (x fastest) with the given box.
int encode_tensor_map_4d(CUtensorMap* map, const void* base, const uint64_t dims[4],
                         const uint64_t strides_bytes[3], const uint32_t box[4]);

}  // namespace how
