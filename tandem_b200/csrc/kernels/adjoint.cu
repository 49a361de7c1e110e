// Instances and launcher of the Lame-parameter gradient kernel.
#include "adjoint.cuh"
#include "dispatch.hpp"

#include "../../../include/tandem_b200.h"

namespace tdg {

namespace {
template <int D, int N>
int run_adj(DevOp<double> const& op, const double* u, const double* p, const double* bcq, const double* dpen,
            double* grad, cudaStream_t s) {
    adjoint_lame_kernel<Shape<D, N, kElasticity>>
        <<<static_cast<unsigned>(op.E), kAdjThreads, 0, s>>>(op, u, p, bcq, dpen, grad);
    return cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
}
template <int D>
int adj_deg(int N, DevOp<double> const& op, const double* u, const double* p, const double* bcq, const double* dpen,
            double* grad, cudaStream_t s) {
    switch (N) {
        case 1: return run_adj<D, 1>(op, u, p, bcq, dpen, grad, s);
        case 2: return run_adj<D, 2>(op, u, p, bcq, dpen, grad, s);
        case 3: return run_adj<D, 3>(op, u, p, bcq, dpen, grad, s);
        case 4: return run_adj<D, 4>(op, u, p, bcq, dpen, grad, s);
        default: return TDG_E_INVALID;
    }
}
}  // namespace

int launch_adjoint_lame(int D, int N, DevOp<double> const& op, const double* u, const double* p, const double* bcq,
                        const double* dpen, double* grad, cudaStream_t s) {
    if (op.E > 0x7fffffff) return TDG_E_INVALID;
    if (D == 2) return adj_deg<2>(N, op, u, p, bcq, dpen, grad, s);
    if (D == 3) return adj_deg<3>(N, op, u, p, bcq, dpen, grad, s);
    return TDG_E_INVALID;
}

}  // namespace tdg

// ------------------------------------------------------------------------------------------------
// Fixed scratch of the allocation-free gradient entry point
// ------------------------------------------------------------------------------------------------

#include <mutex>

namespace tdg {

namespace {
// One copy per device, part of the module image: nothing is allocated when it is used.
static __device__ __align__(256) double g_adjoint_scratch[kAdjointScratchDoubles];
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
double* g_scratch_ptr[kMaxDevices] = {};
}  // namespace

int adjoint_scratch(double** ptr) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TDG_E_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        // once per device, with that device current
        if (cudaGetSymbolAddress(&p, g_adjoint_scratch) != cudaSuccess || !p) return TDG_E_CUDA;
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *ptr = g_scratch_ptr[dev];
    return 0;
}

namespace {
template <int D, int N>
cudaError_t load_adj() {
    cudaFuncAttributes a{};
    return cudaFuncGetAttributes(&a, adjoint_lame_kernel<Shape<D, N, kElasticity>>);
}
}  // namespace

int adjoint_prepare(int D, int N) {
    // Under lazy module loading the module image (and with it the static scratch) and the kernel's
    // code are placed in device memory on first use; doing both here, while the caller is still
    // allowed to allocate, keeps the allocation-free entry point free of them.
    double* p = nullptr;
    if (adjoint_scratch(&p)) return TDG_E_CUDA;
    cudaError_t e = cudaErrorInvalidValue;
    if (D == 2 && N >= 1 && N <= 4) e = N == 1 ? load_adj<2, 1>() : N == 2 ? load_adj<2, 2>() : N == 3 ? load_adj<2, 3>() : load_adj<2, 4>();
    if (D == 3 && N >= 1 && N <= 4) e = N == 1 ? load_adj<3, 1>() : N == 2 ? load_adj<3, 2>() : N == 3 ? load_adj<3, 3>() : load_adj<3, 4>();
    return e == cudaSuccess ? 0 : TDG_E_CUDA;
}

}  // namespace tdg
