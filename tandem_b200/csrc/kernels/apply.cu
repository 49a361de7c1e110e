// Instances and launcher of the operator apply kernel.
#include "apply.cuh"
#include "apply_mma.cuh"
#include "dispatch.hpp"

#include "../../../include/tandem_b200.h"

namespace tdg {

int device_sm_count() {
    static int count = 0;
    if (count == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        if (count <= 0) count = 1;
    }
    return count;
}

namespace {

template <class S, typename T>
int run_apply(DevOp<T> const& op, const T* x, T* y, int nrhs, int64_t ld, cudaStream_t s) {
    using Tl = ApplyTile<S>;
    const size_t smem = sizeof(T) * static_cast<size_t>(apply_smem_elems<S, T>(op.Nq, op.nq));
    static int configured_smem = -1;
    static int blocks_per_sm = 1;
    auto kern = apply_kernel<S, T>;
    if (configured_smem < static_cast<int>(smem)) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)) != cudaSuccess)
            return TDG_E_CUDA;
        configured_smem = static_cast<int>(smem);
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, Tl::NT, smem) != cudaSuccess || nb < 1)
            nb = 1;
        blocks_per_sm = nb;
    }
    const int64_t ntiles = (op.E + Tl::TE - 1) / Tl::TE;
    int64_t grid = static_cast<int64_t>(device_sm_count()) * blocks_per_sm;
    if (grid > ntiles) grid = ntiles;
    if (grid < 1) grid = 1;
    dim3 g(static_cast<unsigned>(grid), static_cast<unsigned>(nrhs));
    kern<<<g, Tl::NT, smem, s>>>(op, x, y, ld);
    return cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
}

template <int D, int N, typename T>
int apply_kind(int kind, DevOp<T> const& op, const T* x, T* y, int nrhs, int64_t ld, cudaStream_t s) {
    if (kind == kPoisson) return run_apply<Shape<D, N, kPoisson>, T>(op, x, y, nrhs, ld, s);
    return run_apply<Shape<D, N, kElasticity>, T>(op, x, y, nrhs, ld, s);
}

template <int D, typename T>
int apply_deg(int N, int kind, DevOp<T> const& op, const T* x, T* y, int nrhs, int64_t ld, cudaStream_t s) {
    switch (N) {
        case 1: return apply_kind<D, 1, T>(kind, op, x, y, nrhs, ld, s);
        case 2: return apply_kind<D, 2, T>(kind, op, x, y, nrhs, ld, s);
        case 3: return apply_kind<D, 3, T>(kind, op, x, y, nrhs, ld, s);
        case 4: return apply_kind<D, 4, T>(kind, op, x, y, nrhs, ld, s);
        default: return TDG_E_INVALID;
    }
}

}  // namespace

template <typename T>
int launch_apply(int D, int N, int kind, DevOp<T> const& op, const T* x, T* y, int nrhs,
                 int64_t ld, cudaStream_t s) {
    if (nrhs < 1) return TDG_E_INVALID;
    if (D == 2) return apply_deg<2, T>(N, kind, op, x, y, nrhs, ld, s);
    if (D == 3) return apply_deg<3, T>(N, kind, op, x, y, nrhs, ld, s);
    return TDG_E_INVALID;
}

namespace {

template <class S>
int run_apply_mma(DevOp<double> const& op, MmaTiles const& mt, const double* x, double* y, int nrhs, int64_t ld,
                  cudaStream_t s, int ctas) {
    using L = MmaTile<S>;
    const MmaLayout lay = mma_layout<S>(op.Nq, op.nq);
    const size_t smem = sizeof(double) * static_cast<size_t>(lay.total);
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem + 2 * L::TE * sizeof(int) > static_cast<size_t>(optin)) return TDG_E_INVALID;
    auto kern = apply_mma_kernel<S>;
    static size_t configured = 0;
    static int per_sm = 1;
    if (configured < smem) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
            cudaSuccess)
            return TDG_E_CUDA;
        configured = smem;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, L::NT, smem) != cudaSuccess || per_sm < 1)
            per_sm = 1;
    }
    const int64_t nwork = static_cast<int64_t>(mt.ntiles) * nrhs;
    const int want = (ctas > 0 && ctas < per_sm) ? ctas : (ctas > 0 ? per_sm : 1);
    int64_t grid = static_cast<int64_t>(device_sm_count()) * want;
    if (grid > nwork) grid = nwork;
    if (grid < 1) grid = 1;
    kern<<<static_cast<unsigned>(grid), L::NT, smem, s>>>(op, mt, x, y, ld, nrhs);
    return cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
}

template <int D, int N>
int mma_kind(int kind, DevOp<double> const& op, MmaTiles const& mt, const double* x, double* y, int nrhs, int64_t ld,
             cudaStream_t s, int ctas) {
    if (kind == kPoisson) return run_apply_mma<Shape<D, N, kPoisson>>(op, mt, x, y, nrhs, ld, s, ctas);
    return run_apply_mma<Shape<D, N, kElasticity>>(op, mt, x, y, nrhs, ld, s, ctas);
}

template <int D>
int mma_deg(int N, int kind, DevOp<double> const& op, MmaTiles const& mt, const double* x, double* y, int nrhs,
            int64_t ld, cudaStream_t s, int ctas) {
    switch (N) {
        case 1: return mma_kind<D, 1>(kind, op, mt, x, y, nrhs, ld, s, ctas);
        case 2: return mma_kind<D, 2>(kind, op, mt, x, y, nrhs, ld, s, ctas);
        case 3: return mma_kind<D, 3>(kind, op, mt, x, y, nrhs, ld, s, ctas);
        case 4: return mma_kind<D, 4>(kind, op, mt, x, y, nrhs, ld, s, ctas);
        default: return TDG_E_INVALID;
    }
}

}  // namespace

int launch_apply_mma(int D, int N, int kind, DevOp<double> const& op, MmaTiles const& mt, const double* x, double* y,
                     int nrhs, int64_t ld, cudaStream_t s, int ctas) {
    if (nrhs < 1 || mt.ntiles < 1) return TDG_E_INVALID;
    if (D == 2) return mma_deg<2>(N, kind, op, mt, x, y, nrhs, ld, s, ctas);
    if (D == 3) return mma_deg<3>(N, kind, op, mt, x, y, nrhs, ld, s, ctas);
    return TDG_E_INVALID;
}

template int launch_apply<double>(int, int, int, DevOp<double> const&, const double*, double*, int,
                                  int64_t, cudaStream_t);
template int launch_apply<float>(int, int, int, DevOp<float> const&, const float*, float*, int,
                                 int64_t, cudaStream_t);

}  // namespace tdg
