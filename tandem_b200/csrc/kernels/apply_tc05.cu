// Instances and launcher of the tcgen05 volume kernel of the FP32 apply (apply_tc05.cuh).
#include "apply_face_tc32.cuh"
#include "apply_tc05.cuh"
#include "dispatch.hpp"

#include <type_traits>

#include "../../../include/tandem_b200.h"

namespace tdg {

namespace {

// The warp-specialised form (vol_tc05p_kernel) or one tile at a time (vol_tc05_kernel).
constexpr bool kTc05Pipelined = true;

template <class S, typename TX, int NP>
int run_vol_tc05(DevOp<float> const& op, Tc32Tiles const& mt, const TX* x, TX* y, int nrhs, int64_t ld,
                 cudaStream_t s) {
    using L = Tc05Vol<S>;
    if (op.Nq > L::NQ || op.Nq < 1 || !mt.tables) return TDG_E_INVALID;
    auto k = kTc05Pipelined ? vol_tc05p_kernel<S, TX, NP> : vol_tc05_kernel<S, TX, NP>;
    static bool conf = false;
    if (!conf) {
        int dev = 0, optin = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (L::BYTES + 1024 > optin) return TDG_E_INVALID;
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES) != cudaSuccess)
            return TDG_E_CUDA;
        conf = true;
    }
    const int64_t nwork = (op.E + L::TE - 1) / L::TE * nrhs;
    int64_t grid = device_sm_count();  // one CTA per SM: the shared memory and half the tensor memory
    if (grid > nwork) grid = nwork;
    if (grid < 1) return 0;
    k<<<static_cast<unsigned>(grid), kTc05Pipelined ? 512 : 256, L::BYTES, s>>>(op, mt.tables, TcfTile<S>::LDT, x, y, ld,
                                                                                 nrhs, mt.status);
    return cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
}

template <int D, int N, typename TX, int NP>
int t5_kind_np(int kind, DevOp<float> const& op, Tc32Tiles const& mt, const TX* x, TX* y, int nrhs, int64_t ld,
               cudaStream_t s) {
    if (kind == kPoisson) return run_vol_tc05<Shape<D, N, kPoisson>, TX, NP>(op, mt, x, y, nrhs, ld, s);
    return run_vol_tc05<Shape<D, N, kElasticity>, TX, NP>(op, mt, x, y, nrhs, ld, s);
}

// passes: 3 (3xTF32) or, for FP64 vectors, 1 (one TF32 pass)
template <int D, int N, typename TX>
int t5_kind(int kind, DevOp<float> const& op, Tc32Tiles const& mt, const TX* x, TX* y, int nrhs, int64_t ld,
            cudaStream_t s, int passes) {
    if (passes == 3) return t5_kind_np<D, N, TX, 3>(kind, op, mt, x, y, nrhs, ld, s);
    if constexpr (std::is_same_v<TX, double>)
        if (passes == 1) return t5_kind_np<D, N, TX, 1>(kind, op, mt, x, y, nrhs, ld, s);
    return TDG_E_INVALID;
}

template <int D, typename TX>
int t5_deg(int N, int kind, DevOp<float> const& op, Tc32Tiles const& mt, const TX* x, TX* y, int nrhs, int64_t ld,
           cudaStream_t s, int passes) {
    switch (N) {
        case 1: return t5_kind<D, 1, TX>(kind, op, mt, x, y, nrhs, ld, s, passes);
        case 2: return t5_kind<D, 2, TX>(kind, op, mt, x, y, nrhs, ld, s, passes);
        case 3: return t5_kind<D, 3, TX>(kind, op, mt, x, y, nrhs, ld, s, passes);
        case 4: return t5_kind<D, 4, TX>(kind, op, mt, x, y, nrhs, ld, s, passes);
        default: return TDG_E_INVALID;
    }
}

}  // namespace

template <typename TX>
int launch_vol_tc05(int D, int N, int kind, DevOp<float> const& op, Tc32Tiles const& mt, const TX* x, TX* y,
                    int nrhs, int64_t ld, cudaStream_t s, int passes) {
    if (nrhs < 1) return TDG_E_INVALID;
    if (D == 2) return t5_deg<2, TX>(N, kind, op, mt, x, y, nrhs, ld, s, passes);
    if (D == 3) return t5_deg<3, TX>(N, kind, op, mt, x, y, nrhs, ld, s, passes);
    return TDG_E_INVALID;
}

template int launch_vol_tc05<float>(int, int, int, DevOp<float> const&, Tc32Tiles const&, const float*, float*, int,
                                    int64_t, cudaStream_t, int);
template int launch_vol_tc05<double>(int, int, int, DevOp<float> const&, Tc32Tiles const&, const double*, double*,
                                     int, int64_t, cudaStream_t, int);

}  // namespace tdg
