// Face-centric FP32 apply on the tensor cores (3xTF32, see apply_tc32.cuh): the split of
// apply_face.cuh -- a volume kernel that stores y and one pass over the facets that evaluates each
// facet's flux once for both sides and adds both lift-backs to y with atomics -- built from the
// tensor-core GEMM helpers of apply_tc32.cuh.  TX is the vectors' type (float, or double for the
// mixed solve: x rounded to FP32 on load, y accumulated in FP64).
#pragma once

#include "apply_face.cuh"
#include "apply_tc32.cuh"
#include "apply_face2.cuh"  // face2_point

namespace tdg {

// One pipeline per CTA, sized for several CTAs per SM.
template <class S>
struct TcfTile {
    static constexpr int TE = tc32_tile_elements(S::D, S::Q);
    static constexpr int NC = TE * S::Q;
    static constexpr int NP = tc_round(NC, 8);
    static constexpr int NTN = NP / 8;
    static constexpr int NPW = tc_npw(NTN);
    static constexpr int NG = NTN / NPW;
    static constexpr int KP = tc_round(S::NBF, 8);
    static constexpr int KS = KP / 8;
    static constexpr int LDT = KP + 4;
    static constexpr int LDU = LDT;
    static constexpr int LDR = tc_ldr(NP);
    static constexpr int MY = tc_round(S::NBF, 16);
    static constexpr int MYT = MY / 16;
    static constexpr int YU = MYT * NG;
    static constexpr int GW = (S::D == 3 && S::Q == 3) ? 6 : 8;
    static constexpr int NW = GW;
    static constexpr int NT = 32 * GW;
    static constexpr int KSP = (YU >= GW) ? 1 : GW / YU;
    static constexpr int UPW = (YU + GW - 1) / GW;
    static constexpr int QCP = (S::D == 3) ? 32 : 64;
    static constexpr int MINB = 2;
};

struct TcfLayoutV {
    int MV, off_U, off_R, total;  // floats
};
template <class S>
__host__ __device__ inline TcfLayoutV tcf_vol_layout(int Nq) {
    using L = TcfTile<S>;
    TcfLayoutV l;
    l.MV = tc_round(S::D * Nq, 16);
    int vrows = tc_round(S::D * L::QCP, 16);
    if (vrows > l.MV) vrows = l.MV;
    int r = vrows * L::LDR;
    if (L::KSP * L::NP * L::MY > r) r = L::KSP * L::NP * L::MY;
    l.off_U = l.MV * L::LDT;
    l.off_R = l.off_U + L::NP * L::LDU;
    l.total = l.off_R + r;
    return l;
}
struct TcfLayoutF {
    int MF, off_TB, off_U0, off_U1, off_R0, off_R1, total;  // floats
};
template <class S>
__host__ __device__ inline TcfLayoutF tcf_face_layout(int nq) {
    using L = TcfTile<S>;
    TcfLayoutF l;
    l.MF = tc_round((S::D + 1) * nq, 16);
    int r = l.MF * L::LDR;
    if (L::KSP * L::NP * L::MY > r) r = L::KSP * L::NP * L::MY;
    l.off_TB = l.MF * L::LDT;
    l.off_U0 = l.off_TB + l.MF * L::LDT;
    l.off_U1 = l.off_U0 + L::NP * L::LDU;
    l.off_R0 = l.off_U1 + L::NP * L::LDU;
    l.off_R1 = l.off_R0 + r;
    l.total = l.off_R1 + r;
    return l;
}

// Writes the k-split Y partials of this warp to st[kp][c][k] (ld MY).
template <class L>
__device__ __forceinline__ void tcf_stage(float* st, const float (&y)[L::UPW][L::NPW][4], int warp, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int kp = warp / L::YU;
    if (kp >= L::KSP) return;
    float* s = st + kp * L::NP * L::MY;
#pragma unroll
    for (int uu = 0; uu < L::UPW; ++uu) {
        const int unit = (warp % L::YU) + uu * L::GW;
        if (unit >= L::YU) break;
        const int myt = unit % L::MYT, ng = unit / L::MYT;
#pragma unroll
        for (int j = 0; j < L::NPW; ++j) {
            const int c = (ng * L::NPW + j) * 8 + 2 * t;
            const int k = myt * 16 + g;
            s[c * L::MY + k] = y[uu][j][0];
            s[(c + 1) * L::MY + k] = y[uu][j][1];
            s[c * L::MY + k + 8] = y[uu][j][2];
            s[(c + 1) * L::MY + k + 8] = y[uu][j][3];
        }
    }
}

template <class S, typename TX, int NP = 3>
__global__ void __launch_bounds__(TcfTile<S>::NT, TcfTile<S>::MINB)
    vol_tc32_kernel(DevOp<float> op, const float* __restrict__ tv, const TX* __restrict__ x, TX* __restrict__ y,
                    int64_t ld, int nrhs) {
    using L = TcfTile<S>;
    constexpr int D = S::D, NBF = S::NBF, Q = S::Q, BS = S::BS, DD = S::DD;
    constexpr int TE = L::TE, NT = L::NT, LDR = L::LDR, LDT = L::LDT, LDU = L::LDU;
    const int Nq = op.Nq;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const TcfLayoutV lay = tcf_vol_layout<S>(Nq);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* sm = reinterpret_cast<float*>(smem_raw);
    float* TV = sm;
    float* sU = sm + lay.off_U;
    float* R0 = sm + lay.off_R;
    __shared__ int s_el[TE];
    for (int i = tid; i < lay.MV * LDT; i += NT) sm[i] = tv[i];

    const int64_t ntiles = (op.E + TE - 1) / TE;
    const int64_t nwork = ntiles * nrhs;
    for (int64_t work = blockIdx.x; work < nwork; work += gridDim.x) {
        int64_t tile, rhs;
        work_tile_rhs(work, ntiles, nrhs, tile, rhs);
        const TX* xr = x + rhs * ld;
        TX* yr = y + rhs * ld;
        __syncthreads();
        if (tid < TE) {
            const int64_t e = tile * TE + tid;
            s_el[tid] = e < op.E ? static_cast<int>(e) : -1;
        }
        __syncthreads();
        for (int i = tid; i < L::NP * L::KP; i += NT) {
            const int c = i / L::KP, k = i % L::KP;
            const int te = c / Q, r = c % Q;
            float v = 0.0f;
            if (k < NBF && c < L::NC && s_el[te] >= 0)
                v = static_cast<float>(xr[static_cast<int64_t>(s_el[te]) * BS + k + NBF * r]);
            sU[c * LDU + k] = v;
        }
        __syncthreads();
        float yacc[L::UPW][L::NPW][4];
#pragma unroll
        for (int a = 0; a < L::UPW; ++a)
#pragma unroll
            for (int j = 0; j < L::NPW; ++j) yacc[a][j][0] = yacc[a][j][1] = yacc[a][j][2] = yacc[a][j][3] = 0.0f;
        for (int q0 = 0; q0 < Nq; q0 += L::QCP) {
            const int nqc = (Nq - q0 < L::QCP) ? (Nq - q0) : L::QCP;
            const int rows = tc_round(nqc * D, 16);
            if (q0 > 0) __syncthreads();
            tc_forward<L, NP>(TV + q0 * D * LDT, sU, R0, TV, sU, R0, 1, rows / 16, warp, lane);
            __syncthreads();
            for (int it = tid; it < TE * nqc; it += NT) {
                const int te = it % TE, qq = it / TE, q = q0 + qq;
                const int el = s_el[te];
                if (el < 0) continue;
                float G[DD];
                const float* vg = op.vG + static_cast<int64_t>(el) * DD * Nq + q;
#pragma unroll
                for (int c = 0; c < DD; ++c) G[c] = vg[c * Nq];
                float* rr = R0 + (qq * D) * LDR + te * Q;
                if constexpr (S::KIND == kPoisson) {
                    const float jwk = op.vCoef[static_cast<int64_t>(el) * Nq + q];
                    float gx[D];
#pragma unroll
                    for (int i = 0; i < D; ++i) {
                        float s = 0.0f;
#pragma unroll
                        for (int a = 0; a < D; ++a) s += G[a * D + i] * rr[a * LDR];
                        gx[i] = jwk * s;
                    }
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        float s = 0.0f;
#pragma unroll
                        for (int i = 0; i < D; ++i) s += G[a * D + i] * gx[i];
                        rr[a * LDR] = s;
                    }
                } else {
                    const float lam = op.vCoef[(static_cast<int64_t>(el) * 2 + 0) * Nq + q];
                    const float mu = op.vCoef[(static_cast<int64_t>(el) * 2 + 1) * Nq + q];
                    float Ju[D][D];
#pragma unroll
                    for (int s = 0; s < D; ++s)
#pragma unroll
                        for (int r = 0; r < D; ++r) {
                            float acc = 0.0f;
#pragma unroll
                            for (int a = 0; a < D; ++a) acc += G[a * D + s] * rr[a * LDR + r];
                            Ju[s][r] = acc;
                        }
                    float div = 0.0f;
#pragma unroll
                    for (int r = 0; r < D; ++r) div += Ju[r][r];
                    float T[D][D];
#pragma unroll
                    for (int uu = 0; uu < D; ++uu) {
                        float sg[D];
#pragma unroll
                        for (int j = 0; j < D; ++j) sg[j] = mu * (Ju[uu][j] + Ju[j][uu]) + ((uu == j) ? lam * div : 0.0f);
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            float s = 0.0f;
#pragma unroll
                            for (int j = 0; j < D; ++j) s += G[a * D + j] * sg[j];
                            T[a][uu] = s;
                        }
                    }
#pragma unroll
                    for (int a = 0; a < D; ++a)
#pragma unroll
                        for (int uu = 0; uu < D; ++uu) rr[a * LDR + uu] = T[a][uu];
                }
            }
            __syncthreads();
            tc_backproject<L, NP>(TV + q0 * D * LDT, R0, yacc, rows, warp, lane);
        }
        __syncthreads();
        tcf_stage<L>(R0, yacc, warp, lane);
        __syncthreads();
        for (int i = tid; i < L::NC * NBF; i += NT) {
            const int c = i / NBF, k = i % NBF;
            const int te = c / Q, r = c % Q;
            const int el = s_el[te];
            if (el < 0) continue;
            float v = 0.0f;
#pragma unroll
            for (int kp = 0; kp < L::KSP; ++kp) v += R0[kp * L::NP * L::MY + c * L::MY + k];
            yr[static_cast<int64_t>(el) * BS + k + NBF * r] = static_cast<TX>(v);
        }
    }
}

// Facet points of the FP32 facet kernel's geometry rows: for 3D elasticity (16 facets per tile, trace
// rows 3 x 56 words apart) the points are stored in quads with the middle two swapped
// (face2_point), so that the two points of a warp's pointwise access are two apart and their trace
// rows fall on disjoint banks; rows per field: nq rounded up to the quad.
template <class S>
__host__ __device__ constexpr bool kTc32PointSwizzle() {
    return S::D == 3 && S::KIND == kElasticity && TcfTile<S>::TE == 16 && TcfTile<S>::LDR % 32 == 24;
}
template <class S>
__host__ __device__ inline int tc32_geo_rows(int nq) {
    return kTc32PointSwizzle<S>() ? (nq + 3) / 4 * 4 : nq;
}

// Coefficient blocks of the facet kernel staged one (side, element) block per warp (true) or by
// one flat index per thread with the padding rewritten every tile (false).
constexpr bool kTc32StageByWarp = true;

template <class S, typename TX, int NP = 3>
__global__ void __launch_bounds__(TcfTile<S>::NT, TcfTile<S>::MINB)
    face_tc32_kernel(DevOp<float> op, const float* __restrict__ tf, FaceTiles ft, const TX* __restrict__ x,
                     TX* __restrict__ y, int64_t ld, int nrhs) {
    using L = TcfTile<S>;
    constexpr int D = S::D, NBF = S::NBF, Q = S::Q, BS = S::BS, DD = S::DD;
    constexpr int TE = L::TE, NT = L::NT, LDR = L::LDR, LDT = L::LDT, LDU = L::LDU;
    constexpr int FF = 2 * D + 2 * DD + (S::KIND == kPoisson ? 0 : 4);  // facet geometry fields
    const int nq = op.nq;
    const int nqg = tc32_geo_rows<S>(nq);  // geometry rows per field
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const TcfLayoutF lay = tcf_face_layout<S>(nq);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* sm = reinterpret_cast<float*>(smem_raw);
    float* TA = sm;
    float* TB = sm + lay.off_TB;
    float* U0 = sm + lay.off_U0;
    float* U1 = sm + lay.off_U1;
    float* R0 = sm + lay.off_R0;
    float* R1 = sm + lay.off_R1;
    // the tile's facet and element ids, double-buffered: the next tile's are loaded during this one
    __shared__ int s_fb[2][TE], s_e0b[2][TE], s_e1b[2][TE];
    const int tab = lay.MF * LDT;

    const int64_t nwork = static_cast<int64_t>(ft.nftiles) * nrhs;
    const int64_t per = (nwork + gridDim.x - 1) / gridDim.x;
    const int64_t w0 = static_cast<int64_t>(blockIdx.x) * per;
    const int64_t w1 = (w0 + per < nwork) ? w0 + per : nwork;
    int cur_a = -1, cur_b = -1;
    if constexpr (kTc32StageByWarp)
        for (int i = tid; i < L::NP * LDU; i += NT) U0[i] = U1[i] = 0.0f;  // padding stays zero
    // {facet, side-0 element, side-1 element} per slot (facet -1 in unused slots) and the tile
    // descriptor: the first tile's now, each next tile's one iteration ahead
    int4 td_next = make_int4(0, 0, 0, 0);
    if (w0 < w1) {
        int64_t t64, r64;
        work_tile_rhs(w0, ft.nftiles, nrhs, t64, r64);
        const int tile0 = static_cast<int>(t64);
        td_next = ft.ftiles[tile0];
        if (tid < TE) {
            const int4 id = ft.tids[static_cast<int64_t>(tile0) * TE + tid];
            s_fb[0][tid] = id.x;
            s_e0b[0][tid] = id.y;
            s_e1b[0][tid] = id.z;
        }
    }
    int sb = 0;
    for (int64_t work = w0; work < w1; ++work, sb ^= 1) {
        int64_t t64, rhs;
        work_tile_rhs(work, ft.nftiles, nrhs, t64, rhs);
        const int tile = static_cast<int>(t64);
        const TX* xr = x + rhs * ld;
        TX* yr = y + rhs * ld;
        const int4 td = td_next;
        const int key = td.z;
        const int l0 = key & 3, l1 = (key >> 2) & 3, mode = key >> 4;
        const bool two = (mode == 1);
        const int* s_f = s_fb[sb];
        const int* s_e0 = s_e0b[sb];
        const int* s_e1 = s_e1b[sb];
        // the next tile's ids and descriptor, in flight during this tile (written to the other
        // buffer at its end, after every read of that buffer in the previous tile)
        int4 id_next = make_int4(-1, -1, -1, 0);
        if (work + 1 < w1) {
            int64_t t1, r1;
            work_tile_rhs(work + 1, ft.nftiles, nrhs, t1, r1);
            const int tile1 = static_cast<int>(t1);
            td_next = ft.ftiles[tile1];
            if (tid < TE) id_next = ft.tids[static_cast<int64_t>(tile1) * TE + tid];
        }
        __syncthreads();  // the previous tile is done; this tile's ids are visible
        if (l0 != cur_a) {
            for (int i = tid; i < tab; i += NT) TA[i] = tf[static_cast<int64_t>(l0) * tab + i];
            cur_a = l0;
        }
        if (two && l1 != cur_b) {
            for (int i = tid; i < tab; i += NT) TB[i] = tf[static_cast<int64_t>(l1) * tab + i];
            cur_b = l1;
        }
        if constexpr (kTc32StageByWarp) {
            // one (side, element) block per warp, the lanes along the block's BS values (all loads
            // of a lane in flight together); the padding (k >= NBF, columns >= NC) stays zero from
            // the start, the columns of empty slots keep stale values that only feed their own
            // (discarded) outputs
            for (int pb = warp; pb < 2 * TE; pb += NT / 32) {
                const int side = pb / TE, te = pb % TE;
                if (side && !two) continue;
                const int e = side ? s_e1[te] : s_e0[te];
                if (s_f[te] < 0 || e < 0) continue;
                const TX* src = xr + static_cast<int64_t>(e) * BS;
                float* dst = (side ? U1 : U0) + te * Q * LDU;
                constexpr int IT = (BS + 31) / 32;
                float v[IT];
#pragma unroll
                for (int j = 0; j < IT; ++j) {
                    const int w = lane + 32 * j;
                    v[j] = w < BS ? static_cast<float>(src[w]) : 0.0f;
                }
#pragma unroll
                for (int j = 0; j < IT; ++j) {
                    const int w = lane + 32 * j;
                    if (w < BS) dst[(w / NBF) * LDU + w % NBF] = v[j];
                }
            }
        } else {
            for (int i = tid; i < L::NP * L::KP; i += NT) {
                const int c = i / L::KP, k = i % L::KP;
                const int te = c / Q, r = c % Q;
                float v0 = 0.0f, v1 = 0.0f;
                if (k < NBF && c < L::NC && s_f[te] >= 0) {
                    v0 = static_cast<float>(xr[static_cast<int64_t>(s_e0[te]) * BS + k + NBF * r]);
                    if (two) v1 = static_cast<float>(xr[static_cast<int64_t>(s_e1[te]) * BS + k + NBF * r]);
                }
                U0[c * LDU + k] = v0;
                if (two) U1[c * LDU + k] = v1;
            }
        }
        __syncthreads();
        tc_forward<L, NP>(TA, U0, R0, TB, U1, R1, two ? 2 : 1, lay.MF / 16, warp, lane);
        __syncthreads();
        for (int it = tid; it < TE * nqg; it += NT) {
            const int te = it % TE, q = kTc32PointSwizzle<S>() ? face2_point(it / TE) : it / TE;
            const int fct = s_f[te];
            if (q >= nq || fct < 0) continue;
            float* ga0p = R0 + (q * D) * LDR + te * Q;
            float* gb0p = R0 + (D * nq + q) * LDR + te * Q;
            float* ga1p = R1 + (q * D) * LDR + te * Q;
            float* gb1p = R1 + (D * nq + q) * LDR + te * Q;
            float u0[Q], u1[Q], g0[D][Q], g1[D][Q];
#pragma unroll
            for (int r = 0; r < Q; ++r) {
                u0[r] = gb0p[r];
                u1[r] = two ? gb1p[r] : 0.0f;
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    g0[a][r] = ga0p[a * LDR + r];
                    g1[a][r] = two ? ga1p[a * LDR + r] : 0.0f;
                }
            }
            if (mode == 3) {
#pragma unroll
                for (int r = 0; r < Q; ++r) {
                    u1[r] = u0[r];
#pragma unroll
                    for (int a = 0; a < D; ++a) g1[a][r] = g0[a][r];
                }
            }
            const float* gp = ft.geo + static_cast<int64_t>(tile) * FF * nqg * TE + it;  // field f at gp[f * fs]
            const int fs = nqg * TE;
            float n[D], nu[D];
#pragma unroll
            for (int i = 0; i < D; ++i) {
                n[i] = gp[i * fs];
                nu[i] = gp[(D + i) * fs];
            }
            const double pen = ft.pen[static_cast<int64_t>(tile) * TE + te];
            const float wq = op.w[q];
            float Gs0[DD], Gs1[DD], cs0[DD], cs1[DD];
            if constexpr (S::KIND == kPoisson) {
#pragma unroll
                for (int c = 0; c < DD; ++c) {
                    cs0[c] = gp[(2 * D + c) * fs];
                    cs1[c] = gp[(2 * D + DD + c) * fs];
                    Gs0[c] = Gs1[c] = 0.0f;
                }
            } else {
#pragma unroll
                for (int c = 0; c < DD; ++c) {
                    Gs0[c] = gp[(2 * D + c) * fs];
                    Gs1[c] = gp[(2 * D + DD + c) * fs];
                }
                cs0[0] = gp[(2 * D + 2 * DD + 0) * fs];
                cs0[1] = gp[(2 * D + 2 * DD + 1) * fs];
                cs1[0] = gp[(2 * D + 2 * DD + 2) * fs];
                cs1[1] = gp[(2 * D + 2 * DD + 3) * fs];
            }
            float ga[D][Q], gb[Q];
            if (mode == 2) {
                facet_lift<S, float>(2, n, nu, pen, wq, u0, g0, u1, g1, Gs0, Gs1, cs0, cs1, ga, gb);
            } else {  // both sides' lift inputs from one averaged stress / flux
                float ha[D][Q], hb[Q];
                if (mode == 3)
                    facet_lift_pair<S, float>(n, nu, pen, wq, u0, g0, u1, g1, Gs0, Gs0, cs0, cs0, ga, gb, ha, hb);
                else
                    facet_lift_pair<S, float>(n, nu, pen, wq, u0, g0, u1, g1, Gs0, Gs1, cs0, cs1, ga, gb, ha, hb);
                if (two) {
#pragma unroll
                    for (int r = 0; r < Q; ++r) {
                        gb1p[r] = hb[r];
#pragma unroll
                        for (int a = 0; a < D; ++a) ga1p[a * LDR + r] = ha[a][r];
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < Q; ++r) {
                gb0p[r] = gb[r];
#pragma unroll
                for (int a = 0; a < D; ++a) ga0p[a * LDR + r] = ga[a][r];
            }
        }
        __syncthreads();
        float y0[L::UPW][L::NPW][4], y1[L::UPW][L::NPW][4];
#pragma unroll
        for (int a = 0; a < L::UPW; ++a)
#pragma unroll
            for (int j = 0; j < L::NPW; ++j)
#pragma unroll
                for (int c = 0; c < 4; ++c) y0[a][j][c] = y1[a][j][c] = 0.0f;
        tc_backproject<L, NP>(TA, R0, y0, lay.MF, warp, lane);
        if (two) tc_backproject<L, NP>(TB, R1, y1, lay.MF, warp, lane);
        __syncthreads();
        tcf_stage<L>(R0, y0, warp, lane);
        if (two) tcf_stage<L>(R1, y1, warp, lane);
        __syncthreads();
        for (int i = tid; i < L::NC * NBF; i += NT) {
            const int c = i / NBF, k = i % NBF;
            const int te = c / Q, r = c % Q;
            if (s_f[te] < 0) continue;
            float v0 = 0.0f, v1 = 0.0f;
#pragma unroll
            for (int kp = 0; kp < L::KSP; ++kp) {
                v0 += R0[kp * L::NP * L::MY + c * L::MY + k];
                if (two) v1 += R1[kp * L::NP * L::MY + c * L::MY + k];
            }
            atomicAdd(&yr[static_cast<int64_t>(s_e0[te]) * BS + k + NBF * r], static_cast<TX>(v0));
            if (two) atomicAdd(&yr[static_cast<int64_t>(s_e1[te]) * BS + k + NBF * r], static_cast<TX>(v1));
        }
        if (tid < TE && work + 1 < w1) {
            s_fb[sb ^ 1][tid] = id_next.x;
            s_e0b[sb ^ 1][tid] = id_next.y;
            s_e1b[sb ^ 1][tid] = id_next.z;
        }
    }
}

}  // namespace tdg
