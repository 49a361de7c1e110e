// Instances and launcher of the software-pipelined face-centric FP64 apply (apply_face2.cuh).
#include "apply_face2.cuh"
#include "dispatch.hpp"

#include "../../../include/tandem_b200.h"

namespace tdg {

namespace {

template <class K>
int configure2(K kern, size_t smem, int threads, int& per_sm) {
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

template <class S, bool ONE>
int run_face2(DevOp<double> const& op, MmaTiles const& mt, FaceTiles const& ft, TileGeo const& tg, const double* x,
              double* y, int nrhs, int64_t ld, cudaStream_t s, int ctas, int qc) {
    using L = MmaTile<S>;
    if (qc < 0 || (qc > 0 && qc % face2_pass_step(S::D) != 0)) return TDG_E_INVALID;
    const Vol2Layout<S> vl = qc == 0 ? vol2_layout_auto<S>(op.Nq) : vol2_layout<S>(op.Nq, qc < op.Nq ? qc : op.Nq);
    // the geometry prefetch where the policy allows it (two CTAs per SM: at most ~113 KB each)
    const size_t two_cta = 112 * 1024;
    int gpre = 0;
    if (kFacetGeometryPrefetch == 2 ||
        (kFacetGeometryPrefetch == 1 && sizeof(double) * face2_layout<S>(op.nq, 1).total <= two_cta))
        gpre = tg.status ? 1 : 0;
    const Face2Layout<S> fl = face2_layout<S>(op.nq, gpre);
    const size_t vsmem = sizeof(double) * static_cast<size_t>(vl.total);
    const size_t fsmem = sizeof(double) * static_cast<size_t>(fl.total);
    auto vk = vol2_kernel<S, ONE>;
    // 3D elasticity: a register-rich facet kernel for one CTA per SM (ctas == 1) besides the
    // two-CTA one
    constexpr bool kTwoVariants = (S::D == 3 && S::Q == 3);
    const bool one = kTwoVariants && ctas == 1;
    auto fk2 = face2_kernel<S, 2, ONE>;
    auto fk1 = face2_kernel<S, kTwoVariants ? 1 : 2, ONE>;
    auto fk = one ? fk1 : fk2;
    static size_t vconf = 0, fconf2 = 0, fconf1 = 0;  // configured dynamic shared memory (grows)
    static int vper = 1, fper2 = 1, fper1 = 1;
    if (vconf < vsmem) {
        if (int rc = configure2(vk, vsmem, L::NT, vper)) return rc;
        vconf = vsmem;
    }
    size_t& fconf = one ? fconf1 : fconf2;
    int& fper = one ? fper1 : fper2;
    if (fconf < fsmem) {
        if (int rc = configure2(fk, fsmem, L::NT, fper)) return rc;
        fconf = fsmem;
    }
    const int sms = device_sm_count();
    const int64_t vwork = (op.E + L::TE - 1) / L::TE * nrhs;
    int64_t vg = static_cast<int64_t>(sms) * ((ctas > 0 && ctas < vper) ? ctas : vper);
    if (vg > vwork) vg = vwork;
    if (vg < 1) vg = 1;
    vk<<<static_cast<unsigned>(vg), L::NT, vsmem, s>>>(op, tg, mt.tables, x, y, ld, nrhs, vl.qc);
    if (cudaGetLastError() != cudaSuccess) return TDG_E_CUDA;
    if (ft.nftiles > 0) {
        const int64_t fwork = static_cast<int64_t>(ft.nftiles) * nrhs;
        int64_t fg = static_cast<int64_t>(sms) * ((ctas > 0 && ctas < fper) ? ctas : fper);
        if (fg > fwork) fg = fwork;
        if (fg < 1) fg = 1;
        fk<<<static_cast<unsigned>(fg), L::NT, fsmem, s>>>(op, ft, tg, x, y, ld, nrhs, gpre);
        if (cudaGetLastError() != cudaSuccess) return TDG_E_CUDA;
    }
    return 0;
}

template <int D, int N>
int face2_kind(int kind, DevOp<double> const& op, MmaTiles const& mt, FaceTiles const& ft, TileGeo const& tg,
               const double* x, double* y, int nrhs, int64_t ld, cudaStream_t s, int ctas, int qc) {
    // one right-hand side: the instances whose work index is the tile itself
    if (kind == kPoisson)
        return nrhs == 1 ? run_face2<Shape<D, N, kPoisson>, true>(op, mt, ft, tg, x, y, nrhs, ld, s, ctas, qc)
                         : run_face2<Shape<D, N, kPoisson>, false>(op, mt, ft, tg, x, y, nrhs, ld, s, ctas, qc);
    return nrhs == 1 ? run_face2<Shape<D, N, kElasticity>, true>(op, mt, ft, tg, x, y, nrhs, ld, s, ctas, qc)
                     : run_face2<Shape<D, N, kElasticity>, false>(op, mt, ft, tg, x, y, nrhs, ld, s, ctas, qc);
}

template <int D>
int face2_deg(int N, int kind, DevOp<double> const& op, MmaTiles const& mt, FaceTiles const& ft, TileGeo const& tg,
              const double* x, double* y, int nrhs, int64_t ld, cudaStream_t s, int ctas, int qc) {
    switch (N) {
        case 1: return face2_kind<D, 1>(kind, op, mt, ft, tg, x, y, nrhs, ld, s, ctas, qc);
        case 2: return face2_kind<D, 2>(kind, op, mt, ft, tg, x, y, nrhs, ld, s, ctas, qc);
        case 3: return face2_kind<D, 3>(kind, op, mt, ft, tg, x, y, nrhs, ld, s, ctas, qc);
        case 4: return face2_kind<D, 4>(kind, op, mt, ft, tg, x, y, nrhs, ld, s, ctas, qc);
        default: return TDG_E_INVALID;
    }
}

}  // namespace

int launch_apply_face2(int D, int N, int kind, DevOp<double> const& op, MmaTiles const& mt, FaceTiles const& ft,
                       TileGeo const& tg, const double* x, double* y, int nrhs, int64_t ld, cudaStream_t s, int ctas,
                       int qc) {
    if (nrhs < 1 || !mt.tables || !tg.vol || (ft.nftiles > 0 && (!tg.fct || !ft.tids))) return TDG_E_INVALID;
    if (D == 2) return face2_deg<2>(N, kind, op, mt, ft, tg, x, y, nrhs, ld, s, ctas, qc);
    if (D == 3) return face2_deg<3>(N, kind, op, mt, ft, tg, x, y, nrhs, ld, s, ctas, qc);
    return TDG_E_INVALID;
}

}  // namespace tdg
