// FP64 throughput probes: the measured FP64 peaks that the roofline of the FP64 apply is quoted
// against (the FP64 CUDA-core FMA pipe and the FP64 tensor pipe in each mma.sync shape sm_100a
// offers for f64).  Each warp keeps kChains independent accumulators so that issue, not latency,
// bounds the loop; the accumulators are written out so that nothing is optimised away.
#include "../../../include/tandem_b200.h"

#include <cuda_runtime.h>

#include <algorithm>

namespace tdg {

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;
constexpr int kUnroll = 4;

__global__ void __launch_bounds__(kThreads) k_peak_dfma(const double* __restrict__ seed, double* __restrict__ out,
                                                        int iters) {
    const double a = seed[0], b = seed[1];
    double c[kChains];
#pragma unroll
    for (int j = 0; j < kChains; ++j) c[j] = seed[2] * (threadIdx.x + j);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int r = 0; r < kUnroll; ++r)
#pragma unroll
            for (int j = 0; j < kChains; ++j) c[j] = fma(c[j], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += c[j];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// mma.sync shapes with f64 operands: m8n8k4 (A 1, B 1, C 2 registers per thread), and the sm_90+
// m16n8k{4,8,16} (A 2/4/8, B 1/2/4, C 4).
template <int SHAPE>
struct MmaF64;

template <>
struct MmaF64<1> {
    static constexpr int kA = 1, kB = 1, kC = 2, kFlops = 2 * 8 * 8 * 4;
    __device__ __forceinline__ static void run(double (&c)[kC], const double (&a)[kA], const double (&b)[kB]) {
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                     : "+d"(c[0]), "+d"(c[1])
                     : "d"(a[0]), "d"(b[0]));
    }
};

template <>
struct MmaF64<2> {
    static constexpr int kA = 2, kB = 1, kC = 4, kFlops = 2 * 16 * 8 * 4;
    __device__ __forceinline__ static void run(double (&c)[kC], const double (&a)[kA], const double (&b)[kB]) {
        asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
                     "{%0,%1,%2,%3};\n"
                     : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                     : "d"(a[0]), "d"(a[1]), "d"(b[0]));
    }
};

template <>
struct MmaF64<3> {
    static constexpr int kA = 4, kB = 2, kC = 4, kFlops = 2 * 16 * 8 * 8;
    __device__ __forceinline__ static void run(double (&c)[kC], const double (&a)[kA], const double (&b)[kB]) {
        asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                     "{%0,%1,%2,%3};\n"
                     : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                     : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
    }
};

template <>
struct MmaF64<4> {
    static constexpr int kA = 8, kB = 4, kC = 4, kFlops = 2 * 16 * 8 * 16;
    __device__ __forceinline__ static void run(double (&c)[kC], const double (&a)[kA], const double (&b)[kB]) {
        asm volatile("mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
                     "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
                     : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                     : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
                       "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
    }
};

template <int SHAPE>
__global__ void __launch_bounds__(kThreads) k_peak_dmma(const double* __restrict__ seed, double* __restrict__ out,
                                                        int iters) {
    using M = MmaF64<SHAPE>;
    double a[M::kA], b[M::kB], c[kChains][M::kC];
#pragma unroll
    for (int i = 0; i < M::kA; ++i) a[i] = seed[0] * (1.0 + 1e-3 * ((threadIdx.x + i) & 7));
#pragma unroll
    for (int i = 0; i < M::kB; ++i) b[i] = seed[1] * (1.0 + 1e-3 * ((threadIdx.x + i) & 3));
#pragma unroll
    for (int j = 0; j < kChains; ++j)
#pragma unroll
        for (int i = 0; i < M::kC; ++i) c[j][i] = 0.0;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < kUnroll; ++r)
#pragma unroll
            for (int j = 0; j < kChains; ++j) M::run(c[j], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < kChains; ++j)
#pragma unroll
        for (int i = 0; i < M::kC; ++i) s += c[j][i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Half the warps on the FMA pipe, half on the tensor pipe (m8n8k4): whether the two FP64 paths
// run concurrently.
__global__ void __launch_bounds__(kThreads) k_peak_both(const double* __restrict__ seed, double* __restrict__ out,
                                                        int iters) {
    const int warp = threadIdx.x >> 5;
    double s = 0.0;
    if (warp & 1) {
        using M = MmaF64<1>;
        double a[1] = {seed[0] * (1.0 + 1e-3 * (threadIdx.x & 7))}, b[1] = {seed[1]}, c[kChains][2] = {};
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int r = 0; r < kUnroll; ++r)
#pragma unroll
                for (int j = 0; j < kChains; ++j) M::run(c[j], a, b);
        }
#pragma unroll
        for (int j = 0; j < kChains; ++j) s += c[j][0] + c[j][1];
    } else {
        const double a = seed[0], b = seed[1];
        double c[kChains];
#pragma unroll
        for (int j = 0; j < kChains; ++j) c[j] = seed[2] * (threadIdx.x + j);
        // 4 x the trips: per trip a tensor warp does 32 m8n8k4 (8,192 FMA), an FMA warp 4 x 32 x
        // 32 = 4,096 FMA, so with separate pipes the FMA half ends first and the rate reads ~1.5 x
        // the tensor pipe's; with one shared pipe it stays at the single-pipe rate
        for (int it = 0; it < iters * 4; ++it) {
#pragma unroll
            for (int r = 0; r < kUnroll; ++r)
#pragma unroll
                for (int j = 0; j < kChains; ++j) c[j] = fma(c[j], a, b);
        }
#pragma unroll
        for (int j = 0; j < kChains; ++j) s += c[j];
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <int SHAPE>
constexpr double dmma_flops_per_warp_iter() {
    return static_cast<double>(MmaF64<SHAPE>::kFlops) * kUnroll * kChains;
}

}  // namespace

}  // namespace tdg

using namespace tdg;

extern "C" int tdg_probe_fp64_peak(int kind, int ctas_per_sm, void* stream, double* tflops) {
    if (!tflops || kind < 0 || kind > 5 || ctas_per_sm < 0 || ctas_per_sm > 8) return TDG_E_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return TDG_E_CUDA;
    const int grid = sms * (ctas_per_sm ? ctas_per_sm : 2);
    double *seed = nullptr, *out = nullptr;
    if (cudaMalloc(&seed, 4 * sizeof(double)) != cudaSuccess) return TDG_E_NOMEM;
    if (cudaMalloc(&out, static_cast<size_t>(grid) * kThreads * sizeof(double)) != cudaSuccess) {
        cudaFree(seed);
        return TDG_E_NOMEM;
    }
    const double hseed[4] = {0.9999999, 1e-7, 1e-3, 0.0};
    cudaMemcpyAsync(seed, hseed, sizeof hseed, cudaMemcpyHostToDevice, s);
    // flops of one launch per loop iteration
    const double warps = static_cast<double>(grid) * (kThreads / 32);
    double per_iter = 0.0;
    switch (kind) {
        case 0: per_iter = static_cast<double>(grid) * kThreads * kUnroll * kChains * 2.0; break;
        case 1: per_iter = warps * dmma_flops_per_warp_iter<1>(); break;
        case 2: per_iter = warps * dmma_flops_per_warp_iter<2>(); break;
        case 3: per_iter = warps * dmma_flops_per_warp_iter<3>(); break;
        case 4: per_iter = warps * dmma_flops_per_warp_iter<4>(); break;
        default:  // half the warps: m8n8k4 per trip; the other half: 4 x the FMA loop per trip
            per_iter = 0.5 * warps * dmma_flops_per_warp_iter<1>() +
                       0.5 * static_cast<double>(grid) * kThreads * kUnroll * kChains * 2.0 * 4.0;
            break;
    }
    // about 20 ms per launch at 40 TFLOP/s
    const int iters = std::max(16, static_cast<int>(8e11 / per_iter));
    auto launch = [&]() {
        switch (kind) {
            case 0: k_peak_dfma<<<grid, kThreads, 0, s>>>(seed, out, iters); break;
            case 1: k_peak_dmma<1><<<grid, kThreads, 0, s>>>(seed, out, iters); break;
            case 2: k_peak_dmma<2><<<grid, kThreads, 0, s>>>(seed, out, iters); break;
            case 3: k_peak_dmma<3><<<grid, kThreads, 0, s>>>(seed, out, iters); break;
            case 4: k_peak_dmma<4><<<grid, kThreads, 0, s>>>(seed, out, iters); break;
            default: k_peak_both<<<grid, kThreads, 0, s>>>(seed, out, iters); break;
        }
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    launch();  // warm-up
    double best = 0.0;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(e0, s);
        launch();
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms > 0.0f) best = std::max(best, per_iter * iters / (ms * 1e-3) / 1e12);
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(seed);
    cudaFree(out);
    if (err != cudaSuccess) return TDG_E_CUDA;
    *tflops = best;
    return 0;
}
