// Vector kernels of the device Krylov solvers.
//
// Vectors are split into *segments*, each with its own Krylov scalars: the right-hand sides of a
// multi-RHS solve (segment r = [r * ld, r * ld + n)) or the independent problems of a block-
// diagonal batch (segment s = the DOF range of problem s).  The host cuts every segment into
// chunks of kChunkMin to kChunk entries (about four per SM over the whole vector); chunk i is
// processed by CTA i, so no CTA straddles two
// segments and a segment's dot product is the sum of its chunks' partial sums (deterministic).
// Every scalar the iteration needs (alpha, beta, residual norms) lives in device memory, one row
// of kScal doubles per segment, so an iteration is a fixed sequence of launches that can be
// captured in a CUDA graph and replayed.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tdg {

constexpr int kScal = 10;
// kRepl flags the segments whose recurrence residual a reliable update replaces; kZQ holds
// z_new . q for the flexible CG step.
enum ScalSlot { kRZ = 0, kPQ = 1, kRZnew = 2, kRR = 3, kActive = 4, kBB = 5, kTmp = 6, kRepl = 7, kZQ = 8 };
constexpr int kVecThreads = 256;
constexpr int64_t kChunk = 32 * 1024;
constexpr int64_t kChunkMin = 1024;

struct Chunk {
    int64_t begin, end;  // entries [begin, end) of the stacked vector
    int seg, pad;
};

__device__ inline double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ inline double block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (wid == 0) {
        s = lane < static_cast<int>(blockDim.x / 32) ? red[lane] : 0.0;
        s = warp_sum(s);
    }
    return s;
}

// partial[chunk][j]: a.b (j = 0) and c.d (j = 1, when c != nullptr) over the chunk.
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_dot2(const Chunk* __restrict__ chunks, const T* __restrict__ a, const T* __restrict__ b,
           const T* __restrict__ c, const T* __restrict__ d, double* __restrict__ partial) {
    const Chunk ch = chunks[blockIdx.x];
    double s0 = 0.0, s1 = 0.0;
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        s0 += static_cast<double>(a[i]) * static_cast<double>(b[i]);
        if (c) s1 += static_cast<double>(c[i]) * static_cast<double>(d[i]);
    }
    __shared__ double red[2][kVecThreads / 32];
    s0 = block_sum(s0, red[0]);
    s1 = block_sum(s1, red[1]);
    if (threadIdx.x == 0) {
        partial[2 * static_cast<int64_t>(blockIdx.x)] = s0;
        partial[2 * static_cast<int64_t>(blockIdx.x) + 1] = s1;
    }
}

// scal[seg][slot_j] = sum of the chunk partials of segment seg (slot < 0: skip).
__global__ void k_dot_finalize(const double* __restrict__ partial, const int* __restrict__ seg_chunk,
                               double* __restrict__ scal, int slot0, int slot1);

// x += alpha p, r -= alpha q with alpha = rz / pq of the segment (inactive: no-op).
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_cg_xr(const Chunk* __restrict__ chunks, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
            const T* __restrict__ q, const double* __restrict__ scal) {
    const Chunk ch = chunks[blockIdx.x];
    const double* s = scal + ch.seg * kScal;
    if (s[kActive] == 0.0) return;
    const double pq = s[kPQ];
    const T alpha = static_cast<T>(pq != 0.0 ? s[kRZ] / pq : 0.0);
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        x[i] += alpha * p[i];
        r[i] -= alpha * q[i];
    }
}

// p = z + beta p with beta = rz_new / rz of the segment (inactive: no-op).  flexible: beta =
// -(z_new . q) / (p . q), the flexible CG step for a preconditioner that varies between
// iterations (Notay, "Flexible conjugate gradients", SIAM J. Sci. Comput. 22, 2000).
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_cg_p(const Chunk* __restrict__ chunks, T* __restrict__ p, const T* __restrict__ z,
           const double* __restrict__ scal, int flexible = 0) {
    const Chunk ch = chunks[blockIdx.x];
    const double* s = scal + ch.seg * kScal;
    if (s[kActive] == 0.0) return;
    const double rz = s[kRZ], pq = s[kPQ];
    const T beta = static_cast<T>(flexible ? (pq != 0.0 ? -s[kZQ] / pq : 0.0) : (rz != 0.0 ? s[kRZnew] / rz : 0.0));
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) p[i] = z[i] + beta * p[i];
}

// rz = rz_new for every active segment (only_replaced: for the active segments flagged kRepl).
__global__ void k_cg_shift(double* __restrict__ scal, int nseg, int only_replaced = 0);

// out = in on the active segments flagged kRepl (with type conversion); other segments untouched.
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kVecThreads)
    k_replace_residual(const Chunk* __restrict__ chunks, const Tin* __restrict__ in, Tout* __restrict__ out,
                       const double* __restrict__ scal) {
    const Chunk ch = chunks[blockIdx.x];
    const double* s = scal + ch.seg * kScal;
    if (s[kActive] == 0.0 || s[kRepl] == 0.0) return;
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) out[i] = static_cast<Tout>(in[i]);
}

// out = in / sqrt(scal[seg][slot]) (type conversion; slot < 0: plain conversion).
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kVecThreads)
    k_scale_convert(const Chunk* __restrict__ chunks, const Tin* __restrict__ in, Tout* __restrict__ out,
                    const double* __restrict__ scal, int slot) {
    const Chunk ch = chunks[blockIdx.x];
    double sc = 1.0;
    if (slot >= 0) {
        const double v = scal[ch.seg * kScal + slot];
        sc = v > 0.0 ? 1.0 / sqrt(v) : 0.0;
    }
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x)
        out[i] = static_cast<Tout>(sc * static_cast<double>(in[i]));
}

// x += sqrt(scal[seg][slot]) d for segments active in `active`.
template <typename Td>
__global__ void __launch_bounds__(kVecThreads)
    k_correct(const Chunk* __restrict__ chunks, double* __restrict__ x, const Td* __restrict__ d,
              const double* __restrict__ scal, int slot, const double* __restrict__ active) {
    const Chunk ch = chunks[blockIdx.x];
    if (active[ch.seg * kScal + kActive] == 0.0) return;
    const double sc = sqrt(scal[ch.seg * kScal + slot]);
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) x[i] += sc * static_cast<double>(d[i]);
}

// r = b - y
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_sub(const Chunk* __restrict__ chunks, const T* __restrict__ b, const T* __restrict__ y, T* __restrict__ r) {
    const Chunk ch = chunks[blockIdx.x];
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) r[i] = b[i] - y[i];
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_copy(const Chunk* __restrict__ chunks, const T* __restrict__ src, T* __restrict__ dst) {
    const Chunk ch = chunks[blockIdx.x];
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) dst[i] = src[i];
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_fill(const Chunk* __restrict__ chunks, T* __restrict__ x, T v) {
    const Chunk ch = chunks[blockIdx.x];
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) x[i] = v;
}

}  // namespace tdg
