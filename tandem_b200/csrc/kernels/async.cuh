// Asynchronous copies into shared memory and mbarrier waits shared by the pipelined kernels:
// cp.async (8 and 16 bytes), the bulk-copy engine (untiled cp.async.bulk, completing on an mbarrier
// transaction count) and bounded waits on an mbarrier phase (a wait that runs out returns false, the
// caller records a status word and gives up instead of spinning on).
#pragma once

#include <cuda_runtime.h>

namespace tdg {

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
// mbarrier-tracked bulk copies (the bulk-copy engine, untiled): one CTA-scope barrier whose
// transaction count the copy completes; waits are bounded (a wait that runs out records a status
// and gives up instead of spinning on).
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// dst[0, bytes) = src[0, bytes) (bytes a multiple of 16, both 16-byte aligned), completing on bar
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// one arrival of this thread on bar (release: this thread's earlier shared-memory writes are
// visible to the threads that see the phase complete)
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for phase `parity` of bar: at most kMaxWaitTries tries and about kMaxWaitNs of wall-clock
// time (the global timer), whichever ends first; false when it ran out.
constexpr int kMaxWaitTries = 1 << 24;
constexpr unsigned long long kMaxWaitNs = 2000000000ull;
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (int i = 0; i < kMaxWaitTries; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63) == 63 && global_ns() - t0 > kMaxWaitNs) return false;
    }
    return false;
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

}  // namespace tdg
