// Bulk copies global -> shared through the TMA unit (cp.async.bulk, no
// tensor map, one destination CTA) completed on an mbarrier, with bounded
// waits.
//
// Rules kept by every user:
//   - source and destination 16-byte aligned, size a multiple of 16 bytes;
//   - the source is this GPU's own memory (never a peer's);
//   - one mbarrier per warp, one copy in flight per barrier, phase tracked
//     by the warp;
//   - every wait is bounded: after kBulkWaitSpins failed polls the caller
//     records an error and waits once more (bounded) for its copy before it
//     stops using the buffer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace vs {

constexpr int kBulkWaitSpins = 1 << 20;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Initialise a barrier expecting one arrival per phase.
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One thread: arm the barrier for `bytes` of transaction and start the copy.
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
    // order earlier generic-proxy accesses of the buffer before the async-proxy write
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
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

// Poll the barrier's phase `parity` at most kBulkWaitSpins times.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (int i = 0; i < kBulkWaitSpins; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

}  // namespace vs
