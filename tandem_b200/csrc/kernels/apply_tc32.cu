// Instances and launcher of the FP32 tensor-core apply (apply_tc32.cuh).
#include "apply_tc32.cuh"
#include "dispatch.hpp"

#include <type_traits>

#include "../../../include/tandem_b200.h"

namespace tdg {

namespace {

template <class S, typename TX, int NP>
int run_apply_tc32(DevOp<float> const& op, Tc32Tiles const& mt, const TX* x, TX* y, int nrhs, int64_t ld,
                   cudaStream_t s, int ctas) {
    using L = Tc32Tile<S>;
    const Tc32Layout lay = tc32_layout<S>(op.Nq, op.nq);
    const size_t smem = sizeof(float) * static_cast<size_t>(lay.total);
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem + 2 * L::TE * sizeof(int) > static_cast<size_t>(optin)) return TDG_E_INVALID;
    auto kern = apply_tc32_kernel<S, TX, NP>;
    static size_t configured = 0;
    static int per_sm = 0;
    if (configured < smem) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
            cudaSuccess)
            return TDG_E_CUDA;
        configured = smem;
        per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, L::NT, smem) != cudaSuccess || per_sm < 1)
            per_sm = 1;
    }
    const int64_t nwork = static_cast<int64_t>(mt.ntiles) * nrhs;
    const int want = (ctas > 0 && ctas < per_sm) ? ctas : per_sm;
    int64_t grid = static_cast<int64_t>(device_sm_count()) * want;
    if (grid > nwork) grid = nwork;
    if (grid < 1) grid = 1;
    kern<<<static_cast<unsigned>(grid), L::NT, smem, s>>>(op, mt, x, y, ld, nrhs);
    return cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
}

template <int D, int N, typename TX, int NP>
int tc_kind_np(int kind, DevOp<float> const& op, Tc32Tiles const& mt, const TX* x, TX* y, int nrhs, int64_t ld,
               cudaStream_t s, int ctas) {
    if (kind == kPoisson) return run_apply_tc32<Shape<D, N, kPoisson>, TX, NP>(op, mt, x, y, nrhs, ld, s, ctas);
    return run_apply_tc32<Shape<D, N, kElasticity>, TX, NP>(op, mt, x, y, nrhs, ld, s, ctas);
}

// passes: 3 (3xTF32) or, for FP64 vectors, 1 (one TF32 pass)
template <int D, int N, typename TX>
int tc_kind(int kind, DevOp<float> const& op, Tc32Tiles const& mt, const TX* x, TX* y, int nrhs, int64_t ld,
            cudaStream_t s, int ctas, int passes) {
    if (passes == 3) return tc_kind_np<D, N, TX, 3>(kind, op, mt, x, y, nrhs, ld, s, ctas);
    if constexpr (std::is_same_v<TX, double>)
        if (passes == 1) return tc_kind_np<D, N, TX, 1>(kind, op, mt, x, y, nrhs, ld, s, ctas);
    return TDG_E_INVALID;
}

template <int D, typename TX>
int tc_deg(int N, int kind, DevOp<float> const& op, Tc32Tiles const& mt, const TX* x, TX* y, int nrhs,
           int64_t ld, cudaStream_t s, int ctas, int passes) {
    switch (N) {
        case 1: return tc_kind<D, 1, TX>(kind, op, mt, x, y, nrhs, ld, s, ctas, passes);
        case 2: return tc_kind<D, 2, TX>(kind, op, mt, x, y, nrhs, ld, s, ctas, passes);
        case 3: return tc_kind<D, 3, TX>(kind, op, mt, x, y, nrhs, ld, s, ctas, passes);
        case 4: return tc_kind<D, 4, TX>(kind, op, mt, x, y, nrhs, ld, s, ctas, passes);
        default: return TDG_E_INVALID;
    }
}

}  // namespace

template <typename TX>
int launch_apply_tc32(int D, int N, int kind, DevOp<float> const& op, Tc32Tiles const& mt, const TX* x, TX* y,
                      int nrhs, int64_t ld, cudaStream_t s, int ctas, int passes) {
    if (nrhs < 1 || mt.ntiles < 1) return TDG_E_INVALID;
    if (D == 2) return tc_deg<2, TX>(N, kind, op, mt, x, y, nrhs, ld, s, ctas, passes);
    if (D == 3) return tc_deg<3, TX>(N, kind, op, mt, x, y, nrhs, ld, s, ctas, passes);
    return TDG_E_INVALID;
}

template int launch_apply_tc32<float>(int, int, int, DevOp<float> const&, Tc32Tiles const&, const float*, float*, int,
                                      int64_t, cudaStream_t, int, int);
template int launch_apply_tc32<double>(int, int, int, DevOp<float> const&, Tc32Tiles const&, const double*, double*,
                                       int, int64_t, cudaStream_t, int, int);

}  // namespace tdg
