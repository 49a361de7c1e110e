// Instances and launcher of the face-centric FP32 apply (apply_face_tc32.cuh).
#include "apply_face_tc32.cuh"
#include "dispatch.hpp"

#include <type_traits>

#include "../../../include/tandem_b200.h"

namespace tdg {

namespace {

template <class K>
int configure_tcf(K kern, size_t smem, int threads, int& per_sm) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem + 1024 > static_cast<size_t>(optin)) return TDG_E_INVALID;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess)
        return TDG_E_CUDA;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return 0;
}

template <class S, typename TX, int NP>
int run_face_tc32(DevOp<float> const& op, Tc32Tiles const& mt, FaceTiles const& ft, const TX* x, TX* y, int nrhs,
                  int64_t ld, cudaStream_t s, int ctas, bool vol) {
    using L = TcfTile<S>;
    const TcfLayoutV vl = tcf_vol_layout<S>(op.Nq);
    const TcfLayoutF fl = tcf_face_layout<S>(op.nq);
    const size_t vsmem = sizeof(float) * static_cast<size_t>(vl.total);
    const size_t fsmem = sizeof(float) * static_cast<size_t>(fl.total);
    auto vk = vol_tc32_kernel<S, TX, NP>;
    auto fk = face_tc32_kernel<S, TX, NP>;
    static size_t vconf = 0, fconf = 0;
    static int vper = 1, fper = 1;
    if (vconf < vsmem) {
        if (int rc = configure_tcf(vk, vsmem, L::NT, vper)) return rc;
        vconf = vsmem;
    }
    if (fconf < fsmem) {
        if (int rc = configure_tcf(fk, fsmem, L::NT, fper)) return rc;
        fconf = fsmem;
    }
    const int sms = device_sm_count();
    const int64_t vwork = (op.E + L::TE - 1) / L::TE * nrhs;
    int64_t vg = static_cast<int64_t>(sms) * ((ctas > 0 && ctas < vper) ? ctas : vper);
    if (vg > vwork) vg = vwork;
    if (vg < 1) vg = 1;
    if (vol) {
        vk<<<static_cast<unsigned>(vg), L::NT, vsmem, s>>>(op, mt.tables, x, y, ld, nrhs);
        if (cudaGetLastError() != cudaSuccess) return TDG_E_CUDA;
    }
    if (ft.nftiles > 0) {
        const int64_t fwork = static_cast<int64_t>(ft.nftiles) * nrhs;
        int64_t fg = static_cast<int64_t>(sms) * ((ctas > 0 && ctas < fper) ? ctas : fper);
        if (fg > fwork) fg = fwork;
        if (fg < 1) fg = 1;
        const float* tf = mt.tables + static_cast<int64_t>(tc_round(S::D * op.Nq, 16)) * L::LDT;
        fk<<<static_cast<unsigned>(fg), L::NT, fsmem, s>>>(op, tf, ft, x, y, ld, nrhs);
        if (cudaGetLastError() != cudaSuccess) return TDG_E_CUDA;
    }
    return 0;
}

template <int D, int N, typename TX, int NP>
int tcf_kind_np(int kind, DevOp<float> const& op, Tc32Tiles const& mt, FaceTiles const& ft, const TX* x, TX* y,
                int nrhs, int64_t ld, cudaStream_t s, int ctas, bool vol) {
    if (kind == kPoisson) return run_face_tc32<Shape<D, N, kPoisson>, TX, NP>(op, mt, ft, x, y, nrhs, ld, s, ctas, vol);
    return run_face_tc32<Shape<D, N, kElasticity>, TX, NP>(op, mt, ft, x, y, nrhs, ld, s, ctas, vol);
}

// passes: 3 (3xTF32) or, for FP64 vectors, 1 (one TF32 pass)
template <int D, int N, typename TX>
int tcf_kind(int kind, DevOp<float> const& op, Tc32Tiles const& mt, FaceTiles const& ft, const TX* x, TX* y,
             int nrhs, int64_t ld, cudaStream_t s, int ctas, bool vol, int passes) {
    if (passes == 3) return tcf_kind_np<D, N, TX, 3>(kind, op, mt, ft, x, y, nrhs, ld, s, ctas, vol);
    if constexpr (std::is_same_v<TX, double>)
        if (passes == 1) return tcf_kind_np<D, N, TX, 1>(kind, op, mt, ft, x, y, nrhs, ld, s, ctas, vol);
    return TDG_E_INVALID;
}

template <int D, typename TX>
int tcf_deg(int N, int kind, DevOp<float> const& op, Tc32Tiles const& mt, FaceTiles const& ft, const TX* x, TX* y,
            int nrhs, int64_t ld, cudaStream_t s, int ctas, bool vol, int passes) {
    switch (N) {
        case 1: return tcf_kind<D, 1, TX>(kind, op, mt, ft, x, y, nrhs, ld, s, ctas, vol, passes);
        case 2: return tcf_kind<D, 2, TX>(kind, op, mt, ft, x, y, nrhs, ld, s, ctas, vol, passes);
        case 3: return tcf_kind<D, 3, TX>(kind, op, mt, ft, x, y, nrhs, ld, s, ctas, vol, passes);
        case 4: return tcf_kind<D, 4, TX>(kind, op, mt, ft, x, y, nrhs, ld, s, ctas, vol, passes);
        default: return TDG_E_INVALID;
    }
}

}  // namespace

template <typename TX>
int launch_apply_face_tc32(int D, int N, int kind, DevOp<float> const& op, Tc32Tiles const& mt, FaceTiles const& ft,
                           const TX* x, TX* y, int nrhs, int64_t ld, cudaStream_t s, int ctas, bool vol05,
                           int passes) {
    if (passes != 3 && passes != 1) return TDG_E_INVALID;
    if (nrhs < 1 || !mt.tables || (ft.nftiles > 0 && (!ft.tids || !ft.geo || !ft.pen))) return TDG_E_INVALID;
    if (D != 2 && D != 3) return TDG_E_INVALID;
    bool vol = true;  // the mma.sync volume kernel, unless the tcgen05 one took the volume term
    if (vol05) {
        const int rc = launch_vol_tc05<TX>(D, N, kind, op, mt, x, y, nrhs, ld, s, passes);
        if (rc && rc != TDG_E_INVALID) return rc;
        vol = rc != 0;
    }
    if (D == 2) return tcf_deg<2, TX>(N, kind, op, mt, ft, x, y, nrhs, ld, s, ctas, vol, passes);
    return tcf_deg<3, TX>(N, kind, op, mt, ft, x, y, nrhs, ld, s, ctas, vol, passes);
}

template int launch_apply_face_tc32<float>(int, int, int, DevOp<float> const&, Tc32Tiles const&, FaceTiles const&,
                                           const float*, float*, int, int64_t, cudaStream_t, int, bool, int);
template int launch_apply_face_tc32<double>(int, int, int, DevOp<float> const&, Tc32Tiles const&, FaceTiles const&,
                                            const double*, double*, int, int64_t, cudaStream_t, int, bool, int);

}  // namespace tdg
