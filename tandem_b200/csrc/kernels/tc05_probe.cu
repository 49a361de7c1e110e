// Known-answer check of the tcgen05 TF32 building blocks (tc05.cuh): one CTA computes
// D[128 x N] = A[128 x K] B[N x K]^T from row-major global operands, staged into the core-matrix
// layout (split into TF32 hi / lo for 3xTF32), one MMA chain into TMEM, a commit to an mbarrier and
// 32x32b loads of the accumulator.  No counterpart in tandem; the parity tests compare it with an
// FP64 product of the same operands before the operator kernels rely on the same descriptors.
#include <cuda_runtime.h>

#include "../../../include/tandem_b200.h"
#include "tc05.cuh"

namespace tdg {
namespace {

__global__ void __launch_bounds__(128) k_tc05_gemm(const float* __restrict__ A, const float* __restrict__ B,
                                                   float* __restrict__ D, int N, int K, int split3, uint32_t cols,
                                                   int* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long bar;
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, warp = tid >> 5;
    // operands 1024-byte aligned inside the dynamic buffer (allocated with 1 KB to spare)
    const uint32_t raw = smem_u32(smem_raw);
    float* Ah = reinterpret_cast<float*>(smem_raw + ((1024u - (raw & 1023u)) & 1023u));
    float* Al = Ah + 128 * K;
    float* Bh = Al + 128 * K;
    float* Bl = Bh + N * K;
    if (warp == 0) {
        tmem_alloc(&tbase, cols);
        tmem_relinquish();
    }
    if (tid == 0) mbar_init(&bar, 1);
    for (int i = tid; i < 128 * K; i += 128) {
        const int r = i / K, k = i % K;
        float h, l;
        split_tf32(A[i], h, l);
        Ah[core_offset(128, r, k)] = h;
        Al[core_offset(128, r, k)] = l;
    }
    for (int i = tid; i < N * K; i += 128) {
        const int r = i / K, k = i % K;
        float h, l;
        split_tf32(B[i], h, l);
        Bh[core_offset(N, r, k)] = h;
        Bl[core_offset(N, r, k)] = l;
    }
    fence_async_smem();
    tc05_fence_before();
    __syncthreads();
    tc05_fence_after();
    const uint32_t tmem = tbase;
    if (tid == 0 && split3 >= 0) {  // split3 < 0: nothing issued, nothing arrives (the bounded wait runs out)
        const uint32_t idesc = idesc_tf32(128, N);
        const uint32_t lboA = (128 / 8) * 128, lboB = static_cast<uint32_t>(N / 8) * 128;
        for (int s = 0; s < K / 8; ++s) {
            const uint32_t offA = 2u * s * lboA, offB = 2u * s * lboB;
            const uint64_t ah = umma_desc(smem_u32(Ah) + offA, lboA, 128), al = umma_desc(smem_u32(Al) + offA, lboA, 128);
            const uint64_t bh = umma_desc(smem_u32(Bh) + offB, lboB, 128), bl = umma_desc(smem_u32(Bl) + offB, lboB, 128);
            umma_tf32(tmem, ah, bh, idesc, s > 0 ? 1u : 0u);
            if (split3) {
                umma_tf32(tmem, ah, bl, idesc, 1u);
                umma_tf32(tmem, al, bh, idesc, 1u);
            }
        }
        umma_commit(&bar);
    }
    const bool done = __all_sync(0xffffffffu, mbar_wait_bounded(&bar, 0));  // warp-uniform for tcgen05.ld
    if (!done && tid == 0) atomicExch(status, 1);
    tc05_fence_after();
    if (done) {
        const int row = 32 * warp + (tid & 31);
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + (static_cast<uint32_t>(32 * warp) << 16) + static_cast<uint32_t>(c0), v);
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i) D[static_cast<int64_t>(row) * N + c0 + i] = v[i];
        }
    }
    tc05_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, cols);
}


// The accumulator's tensor-memory image after D = A[m x k] B[n x k]^T (3xTF32, m = 64 or 128): every
// lane 0..127 and columns 0..2n-1 (pre-filled with -12345) to dump[lane][col].
__global__ void __launch_bounds__(128) k_tc05_layout(const float* __restrict__ A, const float* __restrict__ B,
                                                     float* __restrict__ dump, int M, int N, int K, uint32_t cols,
                                                     int* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long bar;
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t raw = smem_u32(smem_raw);
    float* Ah = reinterpret_cast<float*>(smem_raw + ((1024u - (raw & 1023u)) & 1023u));
    float* Al = Ah + M * K;
    float* Bh = Al + M * K;
    float* Bl = Bh + N * K;
    if (warp == 0) {
        tmem_alloc(&tbase, cols);
        tmem_relinquish();
    }
    if (tid == 0) mbar_init(&bar, 1);
    for (int i = tid; i < M * K; i += 128) {
        const int r = i / K, k = i % K;
        float h, l;
        split_tf32(A[i], h, l);
        Ah[core_offset(M, r, k)] = h;
        Al[core_offset(M, r, k)] = l;
    }
    for (int i = tid; i < N * K; i += 128) {
        const int r = i / K, k = i % K;
        float h, l;
        split_tf32(B[i], h, l);
        Bh[core_offset(N, r, k)] = h;
        Bl[core_offset(N, r, k)] = l;
    }
    fence_async_smem();
    tc05_fence_before();
    __syncthreads();
    tc05_fence_after();
    const uint32_t tmem = tbase;
    const uint32_t lane_base = static_cast<uint32_t>(32 * warp) << 16;
    {  // sentinel in every lane and column the dump reads
        float v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = -12345.0f;
        for (int c0 = 0; c0 < 2 * N; c0 += 16) tmem_st16(tmem + lane_base + static_cast<uint32_t>(c0), v);
        tmem_wait_st();
    }
    tc05_fence_before();
    __syncthreads();
    tc05_fence_after();
    if (tid == 0) {
        const uint32_t idesc = idesc_tf32(M, N);
        const uint32_t lboA = static_cast<uint32_t>(M / 8) * 128, lboB = static_cast<uint32_t>(N / 8) * 128;
        for (int s = 0; s < K / 8; ++s) {
            const uint32_t offA = 2u * s * lboA, offB = 2u * s * lboB;
            const uint64_t ah = umma_desc(smem_u32(Ah) + offA, lboA, 128), al = umma_desc(smem_u32(Al) + offA, lboA, 128);
            const uint64_t bh = umma_desc(smem_u32(Bh) + offB, lboB, 128), bl = umma_desc(smem_u32(Bl) + offB, lboB, 128);
            umma_tf32(tmem, ah, bh, idesc, s > 0 ? 1u : 0u);
            umma_tf32(tmem, ah, bl, idesc, 1u);
            umma_tf32(tmem, al, bh, idesc, 1u);
        }
        umma_commit(&bar);
    }
    const bool done = __all_sync(0xffffffffu, mbar_wait_bounded(&bar, 0));
    if (!done && tid == 0) atomicExch(status, 1);
    tc05_fence_after();
    if (done) {
        const int lanei = 32 * warp + (tid & 31);
        for (int c0 = 0; c0 < 2 * N; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + static_cast<uint32_t>(c0), v);
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i) dump[static_cast<int64_t>(lanei) * 2 * N + c0 + i] = v[i];
        }
    }
    tc05_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, cols);
}
}  // namespace
}  // namespace tdg

extern "C" int tdg_probe_tc05_gemm(const float* A, const float* B, float* D, int n, int k, int split3, void* stream) {
    using namespace tdg;
    if (!A || !B || !D || n < 16 || n > 256 || n % 16 || k < 8 || k > 64 || k % 8 || split3 < -1 || split3 > 1)
        return TDG_E_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t cols = 32;
    while (cols < static_cast<uint32_t>(n)) cols *= 2;
    // operands, 1 KB for the alignment, 4 KB of slack behind the last operand
    const size_t smem = static_cast<size_t>(128 + n) * k * 2 * sizeof(float) + 1024 + 4096;
    if (cudaFuncSetAttribute(k_tc05_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
        cudaSuccess)
        return TDG_E_CUDA;
    int* status = nullptr;
    if (cudaMallocAsync(&status, sizeof(int), s) != cudaSuccess) return TDG_E_NOMEM;
    cudaMemsetAsync(status, 0, sizeof(int), s);
    k_tc05_gemm<<<1, 128, smem, s>>>(A, B, D, n, k, split3, cols, status);
    int rc = cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
    int h = 0;
    if (!rc && cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) rc = TDG_E_CUDA;
    if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = TDG_E_CUDA;
    cudaFreeAsync(status, s);
    if (!rc && h) rc = TDG_E_TIMEOUT;
    return rc;
}

extern "C" int tdg_probe_tc05_layout(const float* A, const float* B, float* dump, int m, int n, int k, void* stream) {
    using namespace tdg;
    if (!A || !B || !dump || (m != 64 && m != 128) || n < 16 || n > 128 || n % 16 || k < 8 || k > 64 || k % 8)
        return TDG_E_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t cols = 32;
    while (cols < static_cast<uint32_t>(2 * n)) cols *= 2;
    const size_t smem = static_cast<size_t>(m + n) * k * 2 * sizeof(float) + 1024 + 4096;
    if (cudaFuncSetAttribute(k_tc05_layout, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
        cudaSuccess)
        return TDG_E_CUDA;
    int* status = nullptr;
    if (cudaMallocAsync(&status, sizeof(int), s) != cudaSuccess) return TDG_E_NOMEM;
    cudaMemsetAsync(status, 0, sizeof(int), s);
    k_tc05_layout<<<1, 128, smem, s>>>(A, B, dump, m, n, k, cols, status);
    int rc = cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
    int h = 0;
    if (!rc && cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) rc = TDG_E_CUDA;
    if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = TDG_E_CUDA;
    cudaFreeAsync(status, s);
    if (!rc && h) rc = TDG_E_TIMEOUT;
    return rc;
}
