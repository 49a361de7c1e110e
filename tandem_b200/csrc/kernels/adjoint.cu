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
