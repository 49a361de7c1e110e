// Instances and launchers of the block-Jacobi kernels.
#include "bjacobi.cuh"
#include "dispatch.hpp"

#include "../../../include/tandem_b200.h"

namespace tdg {

namespace {

template <class S>
int run_assemble(DevOp<double> const& op, double* blk, cudaStream_t s) {
    const size_t smem = sizeof(double) * static_cast<size_t>(bjac_assemble_smem_doubles<S>(op.Nq, op.nq));
    auto kern = bjac_assemble_kernel<S>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
        cudaSuccess)
        return TDG_E_CUDA;
    if (op.E > 0x7fffffff) return TDG_E_INVALID;
    kern<<<static_cast<unsigned>(op.E), 256, smem, s>>>(op, blk);
    return cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
}

template <int D, int N>
int assemble_kind(int kind, DevOp<double> const& op, double* blk, cudaStream_t s) {
    if (kind == kPoisson) return run_assemble<Shape<D, N, kPoisson>>(op, blk, s);
    return run_assemble<Shape<D, N, kElasticity>>(op, blk, s);
}

template <int D>
int assemble_deg(int N, int kind, DevOp<double> const& op, double* blk, cudaStream_t s) {
    switch (N) {
        case 1: return assemble_kind<D, 1>(kind, op, blk, s);
        case 2: return assemble_kind<D, 2>(kind, op, blk, s);
        case 3: return assemble_kind<D, 3>(kind, op, blk, s);
        case 4: return assemble_kind<D, 4>(kind, op, blk, s);
        default: return TDG_E_INVALID;
    }
}

template <int BS, typename T>
int run_invert(int64_t E, const double* blk, T* inv, int* status, cudaStream_t s) {
    const size_t smem = sizeof(double) * (static_cast<size_t>(BS) * BS + BS);
    auto kern = bjac_invert_kernel<BS, T>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
        cudaSuccess)
        return TDG_E_CUDA;
    if (E > 0x7fffffff) return TDG_E_INVALID;
    kern<<<static_cast<unsigned>(E), 256, smem, s>>>(blk, inv, status);
    return cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
}

template <int BS, typename TM, typename TV>
int run_bapply(int64_t E, const TM* inv, const TV* r, TV* z, int nrhs, int64_t ld, cudaStream_t s) {
    constexpr int TE = (256 / BS) > 0 ? (256 / BS) : 1;
    const int64_t ntiles = (E + TE - 1) / TE;
    int64_t grid = static_cast<int64_t>(device_sm_count()) * 8;
    if (grid > ntiles) grid = ntiles;
    if (grid < 1) grid = 1;
    dim3 g(static_cast<unsigned>(grid), static_cast<unsigned>(nrhs));
    bjac_apply_kernel<BS, TM, TV><<<g, 256, 0, s>>>(E, inv, r, z, ld);
    return cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
}

// Block sizes bs = binom(N + D, D) * Q for D in {2, 3}, N in [1, 4], Q in {1, D}.
#define TDG_FOR_EACH_BS(X) \
    X(1) X(2) X(3) X(4) X(6) X(10) X(12) X(15) X(20) X(30) X(35) X(60) X(105)

}  // namespace

int launch_bjac_assemble(int D, int N, int kind, DevOp<double> const& op, double* blk, cudaStream_t s) {
    if (D == 2) return assemble_deg<2>(N, kind, op, blk, s);
    if (D == 3) return assemble_deg<3>(N, kind, op, blk, s);
    return TDG_E_INVALID;
}

template <typename T>
int launch_bjac_invert(int bs, int64_t E, const double* blk, T* inv, int* status, cudaStream_t s) {
    switch (bs) {
#define TDG_CASE(B) \
    case B: return run_invert<B, T>(E, blk, inv, status, s);
        TDG_FOR_EACH_BS(TDG_CASE)
#undef TDG_CASE
        default: return TDG_E_INVALID;
    }
}

template <typename TM, typename TV>
int launch_bjac_apply(int bs, int64_t E, const TM* inv, const TV* r, TV* z, int nrhs, int64_t ld,
                      cudaStream_t s) {
    switch (bs) {
#define TDG_CASE(B) \
    case B: return run_bapply<B, TM, TV>(E, inv, r, z, nrhs, ld, s);
        TDG_FOR_EACH_BS(TDG_CASE)
#undef TDG_CASE
        default: return TDG_E_INVALID;
    }
}

template int launch_bjac_invert<double>(int, int64_t, const double*, double*, int*, cudaStream_t);
template int launch_bjac_invert<float>(int, int64_t, const double*, float*, int*, cudaStream_t);
template int launch_bjac_apply<double, double>(int, int64_t, const double*, const double*, double*, int, int64_t,
                                               cudaStream_t);
template int launch_bjac_apply<float, float>(int, int64_t, const float*, const float*, float*, int, int64_t,
                                             cudaStream_t);
template int launch_bjac_apply<float, double>(int, int64_t, const float*, const double*, double*, int, int64_t,
                                              cudaStream_t);

}  // namespace tdg
