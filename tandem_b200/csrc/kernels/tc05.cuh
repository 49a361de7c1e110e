// 5th-generation tensor cores (tcgen05, sm_100a) for the FP32 operator: TMEM allocation, shared
// memory matrix descriptors of the canonical K-major layout without swizzle, the instruction
// descriptor of kind::tf32 with FP32 accumulation, the MMA issue and its commit to an mbarrier,
// 32x32b loads of the accumulator into registers, and the 3xTF32 split.
//
// Operand layout in shared memory ("core matrices" of 8 rows x 16 bytes): an operand of R rows
// (M for A, N for B; R a multiple of 8) and K 32-bit values per row (K a multiple of 8) is stored
// as [K/4 chunks][R/8 row groups][8 rows][4 values].  The MMA of K step s (8 values, chunks 2s and
// 2s + 1) reads the descriptor that starts at chunk 2s with leading byte offset (between the two K
// chunks) R/8 * 128 and stride byte offset (between row groups) 128.  D[m][n] = sum_k A[m][k]
// B[n][k]: both operands K-major.  The accumulator of an M = 128 MMA holds row m in TMEM lane m and
// column n in TMEM column (base + n); warp w of a warpgroup reads lanes [32 (w % 4), 32 (w % 4) + 32).
#pragma once

#include <cstdint>

#include "async.cuh"

namespace tdg {

// word offset of (row, k) in the core-matrix layout of an operand with R rows
__host__ __device__ constexpr int core_offset(int R, int row, int k) {
    return ((k >> 2) * (R >> 3) + (row >> 3)) * 32 + (row & 7) * 4 + (k & 3);
}

// Shared memory matrix descriptor: start address, leading / stride byte offsets (16-byte units,
// 14 bits each), version 1 (sm_100) at bit 46, base offset 0, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (static_cast<uint64_t>(1) << 46);
}

// Instruction descriptor of kind::tf32: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12 = 2),
// no negation, A and B K-major (bits 15, 16 = 0), N >> 3 at bit 17, M >> 4 at bit 24.  (MN-major
// TF32 operands in the no-swizzle canonical layout gave all-zero products on B200; the kernels use
// K-major operands only.)
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
           (static_cast<uint32_t>(M >> 4) << 24);
}

// D (+)= A B^T, issued by one thread; accumulate = 0 overwrites D
__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// The mbarrier `bar` receives one arrival once every tcgen05 operation this thread issued before
// has completed.
__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc05_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc05_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// generic-proxy writes to shared memory become visible to the tensor core's (async proxy) reads
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// TMEM allocation by one full warp: `cols` (a power of 2, >= 32) columns, base address to *dst
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(dst)), "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(cols) : "memory");
}

// 16 consecutive columns of this thread's TMEM lane (32x32b shape: the warp's 32 lanes)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
// 16 consecutive columns of this thread's TMEM lane from registers
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};\n" ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
        "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
        "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }

// 3xTF32 split: hi keeps the top 10 mantissa bits (round to nearest), lo = x - hi exactly; the tensor
// core reads the top 19 bits of each operand, so hi hi + hi lo + lo hi carries ~2^-21 per product.
__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo) {
    uint32_t h;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(h) : "f"(x));
    hi = __uint_as_float(h);
    lo = x - hi;
}

}  // namespace tdg
