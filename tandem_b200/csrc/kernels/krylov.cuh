// Vector kernels of the device Krylov solvers.  Every scalar the iteration needs (alpha, beta,
// residual norms) lives in device memory, one row of kScal doubles per right-hand side, so an
// iteration is a fixed sequence of launches that can be captured in a CUDA graph and replayed.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tdg {

constexpr int kScal = 8;
enum ScalSlot { kRZ = 0, kPQ = 1, kRZnew = 2, kRR = 3, kActive = 4, kBB = 5, kTmp = 6 };
constexpr int kDotThreads = 256;

__device__ inline double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Partial sums of a.b (and c.d when c != nullptr) per block: partial[(rhs * nb + block) * 2 + j].
template <typename T>
__global__ void __launch_bounds__(kDotThreads)
    k_dot2(int64_t n, int64_t ld, const T* __restrict__ a, const T* __restrict__ b,
           const T* __restrict__ c, const T* __restrict__ d, double* __restrict__ partial) {
    const int rhs = blockIdx.y;
    a += rhs * ld;
    b += rhs * ld;
    if (c) {
        c += rhs * ld;
        d += rhs * ld;
    }
    double s0 = 0.0, s1 = 0.0;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        s0 += static_cast<double>(a[i]) * static_cast<double>(b[i]);
        if (c) s1 += static_cast<double>(c[i]) * static_cast<double>(d[i]);
    }
    __shared__ double red[2][kDotThreads / 32];
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][wid] = s0;
        red[1][wid] = s1;
    }
    __syncthreads();
    if (wid == 0) {
        s0 = lane < kDotThreads / 32 ? red[0][lane] : 0.0;
        s1 = lane < kDotThreads / 32 ? red[1][lane] : 0.0;
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        if (lane == 0) {
            const int64_t o = (static_cast<int64_t>(rhs) * gridDim.x + blockIdx.x) * 2;
            partial[o] = s0;
            partial[o + 1] = s1;
        }
    }
}

// scal[rhs * kScal + slot_j] = sum of the partials of dot j (slot < 0: skip).
__global__ void k_dot_finalize(const double* __restrict__ partial, int nb, double* __restrict__ scal,
                               int slot0, int slot1);

// x += alpha p, r -= alpha q with alpha = rz / pq per right-hand side (inactive: no-op).
template <typename T>
__global__ void k_cg_xr(int64_t n, int64_t ld, T* __restrict__ x, T* __restrict__ r,
                        const T* __restrict__ p, const T* __restrict__ q, const double* __restrict__ scal) {
    const int rhs = blockIdx.y;
    const double* s = scal + rhs * kScal;
    if (s[kActive] == 0.0) return;
    const double pq = s[kPQ];
    const T alpha = static_cast<T>(pq != 0.0 ? s[kRZ] / pq : 0.0);
    const int64_t o = rhs * ld;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        x[o + i] += alpha * p[o + i];
        r[o + i] -= alpha * q[o + i];
    }
}

// p = z + beta p with beta = rz_new / rz (inactive: no-op).
template <typename T>
__global__ void k_cg_p(int64_t n, int64_t ld, T* __restrict__ p, const T* __restrict__ z,
                       const double* __restrict__ scal) {
    const int rhs = blockIdx.y;
    const double* s = scal + rhs * kScal;
    if (s[kActive] == 0.0) return;
    const double rz = s[kRZ];
    const T beta = static_cast<T>(rz != 0.0 ? s[kRZnew] / rz : 0.0);
    const int64_t o = rhs * ld;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        p[o + i] = z[o + i] + beta * p[o + i];
}

// rz = rz_new for every active right-hand side.
__global__ void k_cg_shift(double* __restrict__ scal, int nrhs);

// out = scale[rhs] * in (type conversion), scale = 1 / sqrt(scal[rhs][slot]) or 1 when slot < 0.
template <typename Tin, typename Tout>
__global__ void k_scale_convert(int64_t n, int64_t ld_in, const Tin* __restrict__ in, int64_t ld_out,
                                Tout* __restrict__ out, const double* __restrict__ scal, int slot) {
    const int rhs = blockIdx.y;
    double sc = 1.0;
    if (slot >= 0) {
        const double v = scal[rhs * kScal + slot];
        sc = v > 0.0 ? 1.0 / sqrt(v) : 0.0;
    }
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[rhs * ld_out + i] = static_cast<Tout>(sc * static_cast<double>(in[rhs * ld_in + i]));
}

// x += sqrt(scal[rhs][slot]) * d (mixed precision correction), only for active rhs.
template <typename Td>
__global__ void k_correct(int64_t n, int64_t ld_x, double* __restrict__ x, int64_t ld_d,
                          const Td* __restrict__ d, const double* __restrict__ scal, int slot,
                          const double* __restrict__ active) {
    const int rhs = blockIdx.y;
    if (active && active[rhs * kScal + kActive] == 0.0) return;
    const double sc = sqrt(scal[rhs * kScal + slot]);
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        x[rhs * ld_x + i] += sc * static_cast<double>(d[rhs * ld_d + i]);
}

// r = b - y
template <typename T>
__global__ void k_sub(int64_t n, int64_t ld, const T* __restrict__ b, const T* __restrict__ y,
                      T* __restrict__ r) {
    const int rhs = blockIdx.y;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        r[rhs * ld + i] = b[rhs * ld + i] - y[rhs * ld + i];
}

template <typename T>
__global__ void k_copy(int64_t n, int64_t ld_src, const T* __restrict__ src, int64_t ld_dst,
                       T* __restrict__ dst) {
    const int rhs = blockIdx.y;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[rhs * ld_dst + i] = src[rhs * ld_src + i];
}

template <typename T>
__global__ void k_fill(int64_t n, int64_t ld, T* __restrict__ x, T v) {
    const int rhs = blockIdx.y;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        x[rhs * ld + i] = v;
}

}  // namespace tdg
