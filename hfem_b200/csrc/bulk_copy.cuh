// Bulk asynchronous global -> shared copies on the TMA engine (sm_100a
// cp.async.bulk, untiled, no multicast) with mbarrier transaction counts.
//
// One thread arms a barrier with the byte count of a group of copies
// (arrive.expect_tx) and issues them; every thread then waits on the barrier's
// phase.  Addresses and sizes are multiples of 16 bytes.  Waits are bounded:
// an expired wait returns false and the caller records an error.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace hfem {

constexpr long long BULK_WAIT_LIMIT = 1ll << 24;

__device__ __forceinline__ uint32_t bulk_smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bulk_bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bulk_smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// orders this thread's earlier generic-proxy accesses of shared memory before
// later async-proxy (bulk copy) writes to it
__device__ __forceinline__ void bulk_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void bulk_bar_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bulk_smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     bulk_smem_addr(smem_dst)),
                 "l"(gmem_src), "r"(bytes), "r"(bulk_smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool bulk_bar_wait(uint64_t* bar, uint32_t phase) {
    const uint32_t a = bulk_smem_addr(bar);
    for (long long i = 0; i < BULK_WAIT_LIMIT; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(a), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ bool bulk_aligned(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace hfem
