// Bulk asynchronous copies (cp.async.bulk, the TMA engine; never with cluster
// multicast) into this block's shared memory, counted on mbarriers, and
// bounded waits on those barriers.  Shared by the streamed far-field and
// near-field kernels.  Included by the kernel headers of kernels.cu.
#pragma once

#include <cstdint>

namespace mlfma {
namespace {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(bar),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
constexpr long long kWaitCycles = 1ll << 31;  // about a second at the B200 clock
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, long long limit = kWaitCycles) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}

// Self-check of the bounded wait: one thread waits on a barrier that nothing
// arrives on, for `limit` cycles, and reports 1 in *status when the wait ran
// out (0 if it had completed, which cannot happen).  No copy is in flight, so
// the block exits cleanly and the context stays usable.
__global__ void k_wait_runs_out(long long limit, int* status) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x != 0) return;
    mbar_init(smem_addr(&bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *status = mbar_wait_bounded(smem_addr(&bar), 0, limit) ? 0 : 1;
}
// Global -> this block's shared memory, completion counted on bar (bytes and
// both addresses multiples of 16).
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
}  // namespace
}  // namespace mlfma
