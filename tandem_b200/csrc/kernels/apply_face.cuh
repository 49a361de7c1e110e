// Face-centric FP64 apply on the FP64 tensor pipe: the same operator as apply_mma.cuh split into
// two kernels.
//
//   vol_mma_kernel:  y  = volume term (tandem's apply_volume, app/kernels/elasticity.py:224-229 /
//                         poisson.py:123-128) per element tile; only the volume table is resident,
//                         so several CTAs fit on an SM.
//   face_mma_kernel: y += facet terms.  Each facet with a flux is evaluated once for both sides
//                    (tandem's element-centric apply evaluates every interior facet from both
//                    elements, DGOperator.h:363-396): the two traces R_s = T_{l_s} U_s, the
//                    numerical fluxes of both sides at every facet point (Poisson.cpp:586-631,
//                    Elasticity.cpp:734-801, the side-1 view with swapped coefficients and flipped
//                    normal as Elasticity.cpp:734-747), and the two lift-backs Y_s = T_{l_s}^T L_s,
//                    added to y with atomics.  Facet tiles hold facets with one (local face of side
//                    0, local face of side 1) pair, so a tile uses two face tables; a CTA reloads
//                    them only when the pair changes.
//
// Per interior facet this is 2 trace GEMMs + 2 lift-backs instead of the element-centric 4 + 2.
// The sum over a facet's contributions is unordered (atomics), so results agree with the
// element-centric kernel to rounding, not bit for bit.
#pragma once

#include "apply_mma.cuh"

namespace tdg {

struct FaceTiles {
    const int4* ftiles = nullptr;  // {first index into fperm, count, key, 0}; key = l0 | l1 << 2 | mode << 4
    const int* fperm = nullptr;    // facet ids grouped by key
    const int4* finfo = nullptr;   // per facet: {up0, up1, l0 | l1 << 8, mode}
    const double* tables = nullptr;  // the face tables of the FP64 tensor kernel, [NF][MF][LDT]
    const int4* tids = nullptr;    // per tile slot [ntiles][TE]: {facet, side-0 element, side-1 element
                                   // (-1 unless mode 1), 0}, facet -1 for unused slots
    const float* geo = nullptr;    // FP32 kernel: the tiles' facet geometry [tile][field][nq][TE]
    const double* pen = nullptr;   // FP32 kernel: the tiles' penalties [tile][TE]
    int nftiles = 0;
};

// Facet modes: 1 interior flux, both sides; 2 boundary (Dirichlet / fault) flux, side 0;
// 3 interior flux of side 0 only with the element as its own neighbour (a boundary facet whose
// code is None, as the element-centric apply treats it).

// Lift inputs of the `own` side at one facet point (the numerical flux of SIPG, epsilon = -1):
// ga[a][r] feeds the gradient rows and gb[r] the value row of the lift-back.  n, nu: own outward
// normal (scaled / unit); u0, g0: own trace and reference gradients; u1, g1: the other side's
// (zero for mode 2); G0 / G1: own / other J^-1; c0 / c1: own / other coefficients (Poisson K G
// [DD]; elasticity lam, mu).
// T: the arithmetic (double, or float for the FP32 kernels); the penalty times the jump is formed
// in FP64 and rounded once.
template <class S, typename T>
__device__ __forceinline__ void facet_lift(int mode, const T* n, const T* nu, double pen, T wq, const T (&u0)[S::Q],
                                           const T (&g0)[S::D][S::Q], const T (&u1)[S::Q],
                                           const T (&g1)[S::D][S::Q], const T* G0, const T* G1, const T* c0,
                                           const T* c1, T (&ga)[S::D][S::Q], T (&gb)[S::Q]) {
    constexpr int D = S::D;
    const T half = T(0.5);
    if constexpr (S::KIND == kPoisson) {
        T uh, sg[D];
        if (mode != 2) {
            uh = half * (u1[0] - u0[0]);
            const T pj = static_cast<T>(pen * (static_cast<double>(u0[0]) - static_cast<double>(u1[0])));
#pragma unroll
            for (int p = 0; p < D; ++p) {
                T s = T(0);
#pragma unroll
                for (int a = 0; a < D; ++a) s += c0[a * D + p] * g0[a][0] + c1[a * D + p] * g1[a][0];
                sg[p] = half * s - pj * nu[p];
            }
        } else {
            uh = -u0[0];
            const T pj = static_cast<T>(pen * static_cast<double>(u0[0]));
#pragma unroll
            for (int p = 0; p < D; ++p) {
                T s = T(0);
#pragma unroll
                for (int a = 0; a < D; ++a) s += c0[a * D + p] * g0[a][0];
                sg[p] = s - pj * nu[p];
            }
        }
        T bsum = T(0);
#pragma unroll
        for (int r = 0; r < D; ++r) bsum += n[r] * sg[r];
        gb[0] = -wq * bsum;
#pragma unroll
        for (int a = 0; a < D; ++a) {
            T s = T(0);
#pragma unroll
            for (int r = 0; r < D; ++r) s += n[r] * c0[a * D + r];
            ga[a][0] = wq * uh * s;
        }
    } else {
        const T lam0 = c0[0], mu0 = c0[1], lam1 = c1[0], mu1 = c1[1];
        T sg[D][D];
        {
            T J0[D][D];
#pragma unroll
            for (int s = 0; s < D; ++s)
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    T acc0 = T(0);
#pragma unroll
                    for (int a = 0; a < D; ++a) acc0 += G0[a * D + s] * g0[a][r];
                    J0[s][r] = acc0;
                }
            T d0 = T(0);
#pragma unroll
            for (int r = 0; r < D; ++r) d0 += J0[r][r];
#pragma unroll
            for (int i = 0; i < D; ++i)
#pragma unroll
                for (int j = 0; j < D; ++j) sg[i][j] = mu0 * (J0[i][j] + J0[j][i]) + ((i == j) ? lam0 * d0 : T(0));
        }
        T uhm[D];
        if (mode != 2) {
            T J1[D][D];
#pragma unroll
            for (int s = 0; s < D; ++s)
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    T acc1 = T(0);
#pragma unroll
                    for (int a = 0; a < D; ++a) acc1 += G1[a * D + s] * g1[a][r];
                    J1[s][r] = acc1;
                }
            T d1 = T(0);
#pragma unroll
            for (int r = 0; r < D; ++r) d1 += J1[r][r];
#pragma unroll
            for (int i = 0; i < D; ++i) {
                const T pj = static_cast<T>(pen * (static_cast<double>(u0[i]) - static_cast<double>(u1[i])));
#pragma unroll
                for (int j = 0; j < D; ++j) {
                    const T s1 = mu1 * (J1[i][j] + J1[j][i]) + ((i == j) ? lam1 * d1 : T(0));
                    sg[i][j] = half * (sg[i][j] + s1) - pj * nu[j];
                }
                uhm[i] = half * (u1[i] - u0[i]);
            }
        } else {
#pragma unroll
            for (int i = 0; i < D; ++i) {
                const T pj = static_cast<T>(pen * static_cast<double>(u0[i]));
#pragma unroll
                for (int j = 0; j < D; ++j) sg[i][j] -= pj * nu[j];
                uhm[i] = -u0[i];
            }
        }
        T un = T(0);
#pragma unroll
        for (int r = 0; r < D; ++r) un += uhm[r] * n[r];
#pragma unroll
        for (int uu = 0; uu < D; ++uu) {
            T X[D];
#pragma unroll
            for (int j = 0; j < D; ++j) X[j] = mu0 * (uhm[uu] * n[j] + uhm[j] * n[uu]) + ((uu == j) ? lam0 * un : T(0));
#pragma unroll
            for (int a = 0; a < D; ++a) {
                T s = T(0);
#pragma unroll
                for (int j = 0; j < D; ++j) s += G0[a * D + j] * X[j];
                ga[a][uu] = wq * s;
            }
            T bsum = T(0);
#pragma unroll
            for (int j = 0; j < D; ++j) bsum += n[j] * sg[uu][j];
            gb[uu] = -wq * bsum;
        }
    }
}

// Lift inputs of both sides of an interior facet point (mode 1; mode 3 passes the element's own
// data as side 1): the same values facet_lift gives for side 0 (n, u0 own) and side 1 (-n, u1 own),
// with the averaged stress / flux computed once.  T: the arithmetic (double, or float for the FP32
// kernels); the penalty times the jump is formed in FP64 and rounded once, as in facet_lift.
template <class S, typename T = double>
__device__ __forceinline__ void facet_lift_pair(const T* n, const T* nu, double pen, T wq,
                                                const T (&u0)[S::Q], const T (&g0)[S::D][S::Q],
                                                const T (&u1)[S::Q], const T (&g1)[S::D][S::Q],
                                                const T* G0, const T* G1, const T* c0,
                                                const T* c1, T (&ga0)[S::D][S::Q], T (&gb0)[S::Q],
                                                T (&ga1)[S::D][S::Q], T (&gb1)[S::Q]) {
    constexpr int D = S::D;
    if constexpr (S::KIND == kPoisson) {
        const T uh = T(0.5) * (u1[0] - u0[0]);
        const T pj = static_cast<T>(pen * (static_cast<double>(u0[0]) - static_cast<double>(u1[0])));
        T bsum = T(0);
#pragma unroll
        for (int p = 0; p < D; ++p) {
            T s = T(0);
#pragma unroll
            for (int a = 0; a < D; ++a) s += c0[a * D + p] * g0[a][0] + c1[a * D + p] * g1[a][0];
            bsum += n[p] * (T(0.5) * s - pj * nu[p]);
        }
        gb0[0] = -wq * bsum;
        gb1[0] = wq * bsum;
#pragma unroll
        for (int a = 0; a < D; ++a) {
            T s0 = 0.0, s1 = T(0);
#pragma unroll
            for (int r = 0; r < D; ++r) {
                s0 += n[r] * c0[a * D + r];
                s1 += n[r] * c1[a * D + r];
            }
            ga0[a][0] = wq * uh * s0;
            ga1[a][0] = wq * uh * s1;
        }
    } else {
        const T lam0 = c0[0], mu0 = c0[1], lam1 = c1[0], mu1 = c1[1];
        T sg[D][D];
        {
            T J[D][D];
#pragma unroll
            for (int s = 0; s < D; ++s)
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    T acc = T(0);
#pragma unroll
                    for (int a = 0; a < D; ++a) acc += G0[a * D + s] * g0[a][r];
                    J[s][r] = acc;
                }
            T d = T(0);
#pragma unroll
            for (int r = 0; r < D; ++r) d += J[r][r];
#pragma unroll
            for (int i = 0; i < D; ++i)
#pragma unroll
                for (int j = 0; j < D; ++j) sg[i][j] = mu0 * (J[i][j] + J[j][i]) + ((i == j) ? lam0 * d : T(0));
        }
        {
            T J[D][D];
#pragma unroll
            for (int s = 0; s < D; ++s)
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    T acc = T(0);
#pragma unroll
                    for (int a = 0; a < D; ++a) acc += G1[a * D + s] * g1[a][r];
                    J[s][r] = acc;
                }
            T d = T(0);
#pragma unroll
            for (int r = 0; r < D; ++r) d += J[r][r];
#pragma unroll
            for (int i = 0; i < D; ++i) {
                const T pj = static_cast<T>(pen * (static_cast<double>(u0[i]) - static_cast<double>(u1[i])));
#pragma unroll
                for (int j = 0; j < D; ++j) {
                    const T s1 = mu1 * (J[i][j] + J[j][i]) + ((i == j) ? lam1 * d : T(0));
                    sg[i][j] = T(0.5) * (sg[i][j] + s1) - pj * nu[j];
                }
            }
        }
        T uhm[D];
#pragma unroll
        for (int i = 0; i < D; ++i) uhm[i] = T(0.5) * (u1[i] - u0[i]);
        T un = T(0);
#pragma unroll
        for (int r = 0; r < D; ++r) un += uhm[r] * n[r];
#pragma unroll
        for (int uu = 0; uu < D; ++uu) {
            T X0[D], X1[D];
#pragma unroll
            for (int j = 0; j < D; ++j) {
                const T sym = uhm[uu] * n[j] + uhm[j] * n[uu];
                X0[j] = mu0 * sym + ((uu == j) ? lam0 * un : T(0));
                X1[j] = mu1 * sym + ((uu == j) ? lam1 * un : T(0));
            }
#pragma unroll
            for (int a = 0; a < D; ++a) {
                T s0 = 0.0, s1 = T(0);
#pragma unroll
                for (int j = 0; j < D; ++j) {
                    s0 += G0[a * D + j] * X0[j];
                    s1 += G1[a * D + j] * X1[j];
                }
                ga0[a][uu] = wq * s0;
                ga1[a][uu] = wq * s1;
            }
            T bsum = T(0);
#pragma unroll
            for (int j = 0; j < D; ++j) bsum += n[j] * sg[uu][j];
            gb0[uu] = -wq * bsum;
            gb1[uu] = wq * bsum;
        }
    }
}

// Shared-memory layouts (doubles).
template <class S>
struct VolLayout {
    int MV, off_U, off_R, total;
};
template <class S>
__host__ __device__ inline VolLayout<S> vol_layout(int Nq) {
    using L = MmaTile<S>;
    VolLayout<S> l;
    l.MV = round8(S::D * Nq);
    l.off_U = l.MV * L::LDT;
    l.off_R = l.off_U + L::KP * L::LDN;
    l.total = l.off_R + L::QC * S::D * L::LDN;
    return l;
}
template <class S>
struct FaceLayout {
    int MF, off_TB, off_U0, off_U1, off_R0, off_R1, total;
};
template <class S>
__host__ __device__ inline FaceLayout<S> face_layout(int nq) {
    using L = MmaTile<S>;
    FaceLayout<S> l;
    l.MF = round8((S::D + 1) * nq);
    l.off_TB = l.MF * L::LDT;
    l.off_U0 = l.off_TB + l.MF * L::LDT;
    l.off_U1 = l.off_U0 + L::KP * L::LDN;
    l.off_R0 = l.off_U1 + L::KP * L::LDN;
    l.off_R1 = l.off_R0 + l.MF * L::LDN;
    l.total = l.off_R1 + l.MF * L::LDN;
    return l;
}

template <class S>
__global__ void __launch_bounds__(MmaTile<S>::NT, 2)
    vol_mma_kernel(DevOp<double> op, const double* __restrict__ tv, const double* __restrict__ x,
                   double* __restrict__ y, int64_t ld, int nrhs) {
    using L = MmaTile<S>;
    constexpr int D = S::D, NBF = S::NBF, Q = S::Q, BS = S::BS, DD = S::DD;
    constexpr int TE = L::TE, NT = L::NT, LDN = L::LDN, LDT = L::LDT;
    const int Nq = op.Nq;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const VolLayout<S> lay = vol_layout<S>(Nq);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sm = reinterpret_cast<double*>(smem_raw);
    double* TV = sm;
    double* sU = sm + lay.off_U;
    double* R0 = sm + lay.off_R;
    __shared__ int s_el[TE];
    for (int i = tid; i < lay.MV * LDT; i += NT) sm[i] = tv[i];

    const int64_t ntiles = (op.E + TE - 1) / TE;
    const int64_t nwork = ntiles * nrhs;
    for (int64_t work = blockIdx.x; work < nwork; work += gridDim.x) {
        int64_t tile, rhs;
        work_tile_rhs(work, ntiles, nrhs, tile, rhs);
        const double* xr = x + rhs * ld;
        double* yr = y + rhs * ld;
        __syncthreads();
        if (tid < TE) {
            const int64_t e = tile * TE + tid;
            s_el[tid] = e < op.E ? static_cast<int>(e) : -1;
        }
        __syncthreads();
        for (int i = tid; i < L::KP * L::NP; i += NT) {
            const int k = i / L::NP, c = i % L::NP;
            const int te = c / Q, r = c % Q;
            double v = 0.0;
            if (k < NBF && c < L::NC && s_el[te] >= 0) v = xr[static_cast<int64_t>(s_el[te]) * BS + k + NBF * r];
            sU[k * LDN + c] = v;
        }
        __syncthreads();
        double yacc[L::YPW][2][2];
#pragma unroll
        for (int j = 0; j < L::YPW; ++j) yacc[j][0][0] = yacc[j][0][1] = yacc[j][1][0] = yacc[j][1][1] = 0.0;
        for (int q0 = 0; q0 < Nq; q0 += L::QC) {
            const int nqc = (Nq - q0 < L::QC) ? (Nq - q0) : L::QC;
            const int rows = round8(nqc * D);
            cta_gemm_store<L>(TV + q0 * D * LDT, sU, R0, rows, L::KP / 4, warp, lane);
            __syncthreads();
            for (int it = tid; it < TE * nqc; it += NT) {
                const int te = it % TE, qq = it / TE;
                const int el = s_el[te];
                if (el < 0) continue;
                const int q = q0 + qq;
                double G[DD];
                const double* vg = op.vG + static_cast<int64_t>(el) * DD * Nq + q;
#pragma unroll
                for (int c = 0; c < DD; ++c) G[c] = vg[c * Nq];
                double* rr = R0 + (qq * D) * LDN + te * Q;
                if constexpr (S::KIND == kPoisson) {
                    const double jwk = op.vCoef[static_cast<int64_t>(el) * Nq + q];
                    double gx[D];
#pragma unroll
                    for (int i = 0; i < D; ++i) {
                        double s = 0.0;
#pragma unroll
                        for (int a = 0; a < D; ++a) s += G[a * D + i] * rr[a * LDN];
                        gx[i] = jwk * s;
                    }
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        double s = 0.0;
#pragma unroll
                        for (int i = 0; i < D; ++i) s += G[a * D + i] * gx[i];
                        rr[a * LDN] = s;
                    }
                } else {
                    const double lam = op.vCoef[(static_cast<int64_t>(el) * 2 + 0) * Nq + q];
                    const double mu = op.vCoef[(static_cast<int64_t>(el) * 2 + 1) * Nq + q];
                    double Ju[D][D];
#pragma unroll
                    for (int s = 0; s < D; ++s)
#pragma unroll
                        for (int r = 0; r < D; ++r) {
                            double acc = 0.0;
#pragma unroll
                            for (int a = 0; a < D; ++a) acc += G[a * D + s] * rr[a * LDN + r];
                            Ju[s][r] = acc;
                        }
                    double div = 0.0;
#pragma unroll
                    for (int r = 0; r < D; ++r) div += Ju[r][r];
                    double T[D][D];
#pragma unroll
                    for (int uu = 0; uu < D; ++uu) {
                        double sg[D];
#pragma unroll
                        for (int j = 0; j < D; ++j) sg[j] = mu * (Ju[uu][j] + Ju[j][uu]) + ((uu == j) ? lam * div : 0.0);
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            double s = 0.0;
#pragma unroll
                            for (int j = 0; j < D; ++j) s += G[a * D + j] * sg[j];
                            T[a][uu] = s;
                        }
                    }
#pragma unroll
                    for (int a = 0; a < D; ++a)
#pragma unroll
                        for (int uu = 0; uu < D; ++uu) rr[a * LDN + uu] = T[a][uu];
                }
            }
            __syncthreads();
            cta_gemm_acc_t<L>(TV + q0 * D * LDT, R0, yacc, rows, warp, lane);
            __syncthreads();
        }
        const int g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int j = 0; j < L::YPW; ++j) {
            const int tl = warp + j * L::GW;
            if (tl < L::YT) {
                const int ym = tl % L::MYT, yn = tl / L::MYT;
                const int k = ym * 8 + g;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int c = yn * 8 + 2 * t + h;
                    if (k < NBF && c < L::NC) {
                        const int te = c / Q, r = c % Q;
                        const int el = s_el[te];
                        if (el >= 0) yr[static_cast<int64_t>(el) * BS + k + NBF * r] = yacc[j][0][h] + yacc[j][1][h];
                    }
                }
            }
        }
    }
}

// MINB: CTAs per SM the register budget is sized for (2: 128 registers, which spills a little for
// 3D elasticity; 1: no spills, one CTA per SM).
template <class S, int MINB>
__global__ void __launch_bounds__(MmaTile<S>::NT, MINB)
    face_mma_kernel(DevOp<double> op, FaceTiles ft, const double* __restrict__ x, double* __restrict__ y, int64_t ld,
                    int nrhs) {
    using L = MmaTile<S>;
    constexpr int D = S::D, NBF = S::NBF, Q = S::Q, BS = S::BS, DD = S::DD;
    constexpr int TE = L::TE, NT = L::NT, LDN = L::LDN, LDT = L::LDT;
    const int nq = op.nq;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const FaceLayout<S> lay = face_layout<S>(nq);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sm = reinterpret_cast<double*>(smem_raw);
    double* TA = sm;
    double* TB = sm + lay.off_TB;
    double* U0 = sm + lay.off_U0;
    double* U1 = sm + lay.off_U1;
    double* R0 = sm + lay.off_R0;
    double* R1 = sm + lay.off_R1;
    __shared__ int s_f[TE], s_e0[TE], s_e1[TE];
    const int tab = lay.MF * LDT;

    // contiguous work ranges per CTA keep the table pair mostly unchanged
    const int64_t nwork = static_cast<int64_t>(ft.nftiles) * nrhs;
    const int64_t per = (nwork + gridDim.x - 1) / gridDim.x;
    const int64_t w0 = static_cast<int64_t>(blockIdx.x) * per;
    const int64_t w1 = (w0 + per < nwork) ? w0 + per : nwork;
    int cur_a = -1, cur_b = -1;  // face tables held in TA / TB
    for (int64_t work = w0; work < w1; ++work) {
        int64_t t64, rhs;
        work_tile_rhs(work, ft.nftiles, nrhs, t64, rhs);
        const int tile = static_cast<int>(t64);
        const double* xr = x + rhs * ld;
        double* yr = y + rhs * ld;
        const int4 td = ft.ftiles[tile];
        const int key = td.z;
        const int l0 = key & 3, l1 = (key >> 2) & 3, mode = key >> 4;
        const bool two = (mode == 1);
        __syncthreads();
        if (l0 != cur_a) {
            for (int i = tid; i < tab; i += NT) TA[i] = ft.tables[static_cast<int64_t>(l0) * tab + i];
            cur_a = l0;
        }
        if (two && l1 != cur_b) {
            for (int i = tid; i < tab; i += NT) TB[i] = ft.tables[static_cast<int64_t>(l1) * tab + i];
            cur_b = l1;
        }
        if (tid < TE) {
            int f = -1, e0 = -1, e1 = -1;
            if (tid < td.y) {
                f = ft.fperm[td.x + tid];
                const int4 fi = ft.finfo[f];
                e0 = fi.x;
                e1 = fi.y;
            }
            s_f[tid] = f;
            s_e0[tid] = e0;
            s_e1[tid] = e1;
        }
        __syncthreads();
        for (int i = tid; i < L::KP * L::NP; i += NT) {
            const int k = i / L::NP, c = i % L::NP;
            const int te = c / Q, r = c % Q;
            double v0 = 0.0, v1 = 0.0;
            if (k < NBF && c < L::NC && s_f[te] >= 0) {
                v0 = xr[static_cast<int64_t>(s_e0[te]) * BS + k + NBF * r];
                if (two) v1 = xr[static_cast<int64_t>(s_e1[te]) * BS + k + NBF * r];
            }
            U0[k * LDN + c] = v0;
            if (two) U1[k * LDN + c] = v1;
        }
        __syncthreads();
        if (two)
            cta_gemm_store2<L>(TA, U0, R0, TB, U1, R1, lay.MF, L::KP / 4, warp, lane);
        else
            cta_gemm_store<L>(TA, U0, R0, lay.MF, L::KP / 4, warp, lane);
        __syncthreads();
        for (int it = tid; it < TE * nq; it += NT) {
            const int te = it % TE, q = it / TE;
            const int fct = s_f[te];
            if (fct < 0) continue;
            double* ga0p = R0 + (q * D) * LDN + te * Q;
            double* gb0p = R0 + (D * nq + q) * LDN + te * Q;
            double* ga1p = R1 + (q * D) * LDN + te * Q;
            double* gb1p = R1 + (D * nq + q) * LDN + te * Q;
            double u0[Q], u1[Q], g0[D][Q], g1[D][Q];
#pragma unroll
            for (int r = 0; r < Q; ++r) {
                u0[r] = gb0p[r];
                u1[r] = two ? gb1p[r] : 0.0;
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    g0[a][r] = ga0p[a * LDN + r];
                    g1[a][r] = two ? ga1p[a * LDN + r] : 0.0;
                }
            }
            if (mode == 3) {  // own neighbour: the other side is the element itself
#pragma unroll
                for (int r = 0; r < Q; ++r) {
                    u1[r] = u0[r];
#pragma unroll
                    for (int a = 0; a < D; ++a) g1[a][r] = g0[a][r];
                }
            }
            double n[D], nu[D], mn[D], mnu[D];
#pragma unroll
            for (int i = 0; i < D; ++i) {
                n[i] = op.fN[(static_cast<int64_t>(fct) * D + i) * nq + q];
                nu[i] = op.fNunit[(static_cast<int64_t>(fct) * D + i) * nq + q];
                mn[i] = -n[i];
                mnu[i] = -nu[i];
            }
            const double pen = op.penalty[fct];
            const double wq = op.w[q];
            double Gs0[DD], Gs1[DD], cs0[DD], cs1[DD];
            if constexpr (S::KIND == kPoisson) {
                const double* kg = op.fCoef + static_cast<int64_t>(fct) * 2 * DD * nq + q;
#pragma unroll
                for (int c = 0; c < DD; ++c) {
                    cs0[c] = kg[(0 * DD + c) * nq];
                    cs1[c] = kg[(1 * DD + c) * nq];
                    Gs0[c] = Gs1[c] = 0.0;
                }
            } else {
                const double* gg = op.fG + static_cast<int64_t>(fct) * 2 * DD * nq + q;
#pragma unroll
                for (int c = 0; c < DD; ++c) {
                    Gs0[c] = gg[(0 * DD + c) * nq];
                    Gs1[c] = gg[(1 * DD + c) * nq];
                }
                const double* lm = op.fCoef + static_cast<int64_t>(fct) * 4 * nq + q;
                cs0[0] = lm[0 * nq];
                cs0[1] = lm[1 * nq];
                cs1[0] = lm[2 * nq];
                cs1[1] = lm[3 * nq];
            }
            {
                // side 0 (for mode 3, side 1's data are side 0's, as the element-centric apply
                // reads them for a facet whose neighbour is the element itself); the inputs stay
                // in registers, so the lift inputs can overwrite the traces right away
                double ga[D][Q], gb[Q];
                if (mode == 3)
                    facet_lift<S, double>(1, n, nu, pen, wq, u0, g0, u1, g1, Gs0, Gs0, cs0, cs0, ga, gb);
                else
                    facet_lift<S, double>(mode, n, nu, pen, wq, u0, g0, u1, g1, Gs0, Gs1, cs0, cs1, ga, gb);
#pragma unroll
                for (int r = 0; r < Q; ++r) {
                    gb0p[r] = gb[r];
#pragma unroll
                    for (int a = 0; a < D; ++a) ga0p[a * LDN + r] = ga[a][r];
                }
            }
            if (two) {
                double ha[D][Q], hb[Q];
                facet_lift<S, double>(1, mn, mnu, pen, wq, u1, g1, u0, g0, Gs1, Gs0, cs1, cs0, ha, hb);
#pragma unroll
                for (int r = 0; r < Q; ++r) {
                    gb1p[r] = hb[r];
#pragma unroll
                    for (int a = 0; a < D; ++a) ga1p[a * LDN + r] = ha[a][r];
                }
            }
        }
        __syncthreads();
        double y0[L::YPW][2][2], y1[L::YPW][2][2];
#pragma unroll
        for (int j = 0; j < L::YPW; ++j)
#pragma unroll
            for (int a = 0; a < 2; ++a) y0[j][a][0] = y0[j][a][1] = y1[j][a][0] = y1[j][a][1] = 0.0;
        cta_gemm_acc_t<L>(TA, R0, y0, lay.MF, warp, lane);
        if (two) cta_gemm_acc_t<L>(TB, R1, y1, lay.MF, warp, lane);
        const int g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int j = 0; j < L::YPW; ++j) {
            const int tl = warp + j * L::GW;
            if (tl < L::YT) {
                const int ym = tl % L::MYT, yn = tl / L::MYT;
                const int k = ym * 8 + g;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int c = yn * 8 + 2 * t + h;
                    if (k < NBF && c < L::NC) {
                        const int te = c / Q, r = c % Q;
                        if (s_f[te] >= 0) {
                            atomicAdd(&yr[static_cast<int64_t>(s_e0[te]) * BS + k + NBF * r], y0[j][0][h] + y0[j][1][h]);
                            if (two)
                                atomicAdd(&yr[static_cast<int64_t>(s_e1[te]) * BS + k + NBF * r],
                                          y1[j][0][h] + y1[j][1][h]);
                        }
                    }
                }
            }
        }
    }
}

}  // namespace tdg
