// Instances and launchers of the fault kernels (Poisson).
#include "dispatch.hpp"
#include "fault.cuh"

#include "../../../include/tandem_b200.h"

namespace tdg {

namespace {

template <int D, int N>
int run_fault(bool traction, DevOp<double> const& op, DevFault const& fl, const double* u, int64_t ld,
              const double* slip, int64_t ld_slip, double* out, int64_t ld_out, int nrhs, cudaStream_t s) {
    using S = Shape<D, N, kPoisson>;
    dim3 grid(static_cast<unsigned>(fl.nfault), static_cast<unsigned>(nrhs));
    if (traction)
        fault_traction_kernel<S><<<grid, kFaultThreads, 0, s>>>(op, fl, u, ld, slip, ld_slip, out, ld_out);
    else
        fault_rhs_kernel<S><<<grid, kFaultThreads, 0, s>>>(op, fl, slip, ld_slip, out, ld_out);
    return cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
}

template <int D>
int fault_deg(int N, bool traction, DevOp<double> const& op, DevFault const& fl, const double* u, int64_t ld,
              const double* slip, int64_t ld_slip, double* out, int64_t ld_out, int nrhs, cudaStream_t s) {
    switch (N) {
        case 1: return run_fault<D, 1>(traction, op, fl, u, ld, slip, ld_slip, out, ld_out, nrhs, s);
        case 2: return run_fault<D, 2>(traction, op, fl, u, ld, slip, ld_slip, out, ld_out, nrhs, s);
        case 3: return run_fault<D, 3>(traction, op, fl, u, ld, slip, ld_slip, out, ld_out, nrhs, s);
        case 4: return run_fault<D, 4>(traction, op, fl, u, ld, slip, ld_slip, out, ld_out, nrhs, s);
        default: return TDG_E_INVALID;
    }
}

}  // namespace

int launch_fault(int D, int N, bool traction, DevOp<double> const& op, DevFault const& fl, const double* u,
                 int64_t ld, const double* slip, int64_t ld_slip, double* out, int64_t ld_out, int nrhs,
                 cudaStream_t s) {
    if (nrhs < 1 || nrhs > 65535 || fl.nfault < 1 || op.nq > kFaultMaxQ) return TDG_E_INVALID;
    if (D == 2) return fault_deg<2>(N, traction, op, fl, u, ld, slip, ld_slip, out, ld_out, nrhs, s);
    if (D == 3) return fault_deg<3>(N, traction, op, fl, u, ld, slip, ld_slip, out, ld_out, nrhs, s);
    return TDG_E_INVALID;
}

}  // namespace tdg
