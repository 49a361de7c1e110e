// FP64 operator apply on the FP64 tensor pipe (mma.sync m8n8k4 .f64).
//
// Same algorithm as apply.cuh (tandem's element-centric apply: volume term, then per local face
// the own and neighbour traces, numerical fluxes and lift-back; see the citations there), written
// as a sequence of CTA-wide small GEMMs over a tile of TE elements whose columns are
// (element, component) pairs:
//
//   volume, per chunk of QC volume points:
//     R = TV[chunk] x U              reference gradients at the points        (M = QC*D, K = Nbf)
//     R <- pointwise stress/flux      (SIMT, per element and point)
//     Y += TV[chunk]^T x R            back-projection                          (K = QC*D)
//   per local face f:
//     R0 = TF[f] x U, R1 = TF[l'] x Un  own / neighbour traces (gradients and values)
//     R0 <- lift inputs from the numerical fluxes (SIMT)
//     Y += TF[f]^T x R0
//
// TV / TF are the basis-derivative and basis-value tables at the volume / facet points, resident
// in shared memory for the lifetime of the (persistent) CTA.  l' is the neighbour's local face
// number; elements are grouped into tiles with one neighbour-face signature, so every GEMM of a
// tile uses a single table (host side: build_tiles in capi.cu).  Y lives in mma accumulator
// fragments; nothing is accumulated through memory, there are no atomics, and each output block
// is written once.  The kernel can run several independent tile pipelines per CTA (own buffers,
// named barriers, shared tables; mma_pipelines), so one pipeline's global-memory waits overlap
// another's tensor work.
//
// Shared-memory leading dimensions are congruent to 4 or 12 mod 16 doubles, which makes the
// 8x4 / 4x8 fragment loads of a half warp hit 16 distinct 8-byte bank pairs.
#pragma once

#include "common.cuh"

namespace tdg {

// Smallest leading dimension >= n congruent to 4 or 12 modulo 16 (doubles): the 8x4 / 4x8
// fragment loads of a half warp then hit 16 distinct 8-byte bank pairs.
__host__ __device__ constexpr int mma_ld(int n) {
    return (n % 16 <= 4) ? (n - n % 16 + 4) : ((n % 16 <= 12) ? (n - n % 16 + 12) : (n - n % 16 + 20));
}
// Elements per tile (24 columns) and tile pipelines per CTA.  Two pipelines fit the shared memory
// of 3D p4 elasticity only with 4-element tiles (12 of 16 mma columns used); measured on B200 that
// runs 7.14 ms against 6.75 ms for one pipeline of 8-element tiles, so every shape uses one.
__host__ __device__ constexpr int mma_tile_elements(int D, int N, int Q) {
    return (D > 0 && N > 0) ? (24 + Q - 1) / Q : 0;
}
__host__ __device__ constexpr int mma_pipelines(int D, int N, int Q) { return (D > 0 && N > 0 && Q > 0) ? 1 : 0; }

// Layout parameters shared by the host (table packing, tiling) and the kernel.
template <class S>
struct MmaTile {
    static constexpr int NT = 256, NW = 8;
    static constexpr int NGRP = mma_pipelines(S::D, S::N, S::Q);   // tile pipelines per CTA
    static constexpr int GW = NW / NGRP, GT = 32 * GW;             // warps / threads per pipeline
    static constexpr int TE = mma_tile_elements(S::D, S::N, S::Q); // elements per tile
    static constexpr int NC = TE * S::Q;                           // used columns
    static constexpr int NP = (NC + 7) / 8 * 8;                    // padded columns
    static constexpr int NTN = NP / 8;                             // n-tiles
    static constexpr int KP = (S::NBF + 3) / 4 * 4;                // padded Nbf (K of R = T x U)
    static constexpr int MY = (S::NBF + 7) / 8 * 8;                // padded Nbf (M of Y)
    static constexpr int MYT = MY / 8;                             // m-tiles of Y
    static constexpr int YT = MYT * NTN;                           // Y tiles
    static constexpr int YPW = (YT + GW - 1) / GW;                 // Y tiles per warp
    // Y's A^T fragments read table columns up to MY - 1 >= KP: those extra columns fall into the
    // next table row (finite values) and only feed Y rows >= NBF, which are never written.
    static constexpr int LDT = mma_ld(KP);
    static constexpr int LDN = mma_ld(NP);
    static constexpr int QC = 24;                                  // volume points per chunk (QC*D % 8 == 0)
};

__host__ __device__ inline int round8(int x) { return (x + 7) / 8 * 8; }

struct MmaLayout {
    int MV, MF;           // padded rows of TV and of each TF
    int off_TF;           // tables: TV at 0, TF at off_TF (doubles)
    int off_grp, grp;     // first pipeline buffer, doubles per pipeline
    int off_U, off_UN, off_R0, off_R1;  // offsets inside a pipeline's buffers
    int total;            // doubles
};

template <class S>
__host__ __device__ inline MmaLayout mma_layout(int Nq, int nq) {
    using L = MmaTile<S>;
    MmaLayout l;
    l.MV = round8(S::D * Nq);
    l.MF = round8((S::D + 1) * nq);
    int rv = L::QC * S::D;
    int mr = l.MF > rv ? l.MF : rv;
    l.off_TF = l.MV * L::LDT;
    l.off_grp = l.off_TF + S::NF * l.MF * L::LDT;
    l.off_U = 0;
    l.off_UN = l.off_U + L::KP * L::LDN;
    l.off_R0 = l.off_UN + L::KP * L::LDN;
    l.off_R1 = l.off_R0 + mr * L::LDN;
    l.grp = l.off_R1 + l.MF * L::LDN;
    l.total = l.off_grp + L::NGRP * l.grp;
    return l;
}

struct MmaTiles {
    const int4* tiles = nullptr;  // {first index into perm, count, signature, 0}
    const int* perm = nullptr;    // element ids grouped by signature
    const double* tables = nullptr;  // TV then TF[0..NF-1], packed as in shared memory
    int ntiles = 0;
    int table_doubles = 0;
};

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// C[M x NP] = A[M x K] B[K x NP] for rows [0, mrows): A rows from `A` (ld LDT), B from `B` (ld
// LDN), result to `C` (ld LDN).  The (m, n) output tiles are dealt round-robin to the warps; a
// warp advances up to four of its tiles together so that consecutive mma have independent
// accumulators.
template <class L>
__device__ __forceinline__ void cta_gemm_store(const double* A, const double* B, double* C, int mrows, int ksteps,
                                               int warp, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int ntiles = (mrows / 8) * L::NTN;
    for (int t0 = warp; t0 < ntiles; t0 += 4 * L::GW) {
        double acc[4][2];
        const double* ap[4];
        const double* bp[4];
        int cnt = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            acc[j][0] = acc[j][1] = 0.0;
            const int tile = t0 + j * L::GW;
            const int tt = tile < ntiles ? tile : t0;
            const int mt = tt / L::NTN, nt = tt % L::NTN;
            ap[j] = A + (mt * 8 + g) * L::LDT + t;
            bp[j] = B + t * L::LDN + nt * 8 + g;
            cnt += tile < ntiles;
        }
        for (int ks = 0; ks < ksteps; ++ks) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (j < cnt) dmma(acc[j], ap[j][ks * 4], bp[j][ks * 4 * L::LDN]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (j < cnt) {
                const int tile = t0 + j * L::GW;
                const int mt = tile / L::NTN, nt = tile % L::NTN;
                double* c = C + (mt * 8 + g) * L::LDN + nt * 8 + 2 * t;
                c[0] = acc[j][0];
                c[1] = acc[j][1];
            }
        }
    }
}

// Two independent GEMMs C0 = A0 B0 and C1 = A1 B1 of the same shape, dealt to the warps as one
// tile space (better balance than two separate passes).
template <class L>
__device__ __forceinline__ void cta_gemm_store2(const double* A0, const double* B0, double* C0, const double* A1,
                                                const double* B1, double* C1, int mrows, int ksteps, int warp,
                                                int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int per = (mrows / 8) * L::NTN;
    const int ntiles = 2 * per;
    for (int t0 = warp; t0 < ntiles; t0 += 4 * L::GW) {
        double acc[4][2];
        const double* ap[4];
        const double* bp[4];
        int cnt = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            acc[j][0] = acc[j][1] = 0.0;
            const int tile = t0 + j * L::GW;
            const int tt = tile < ntiles ? tile : t0;
            const int which = tt / per, loc = tt % per;
            const int mt = loc / L::NTN, nt = loc % L::NTN;
            ap[j] = (which ? A1 : A0) + (mt * 8 + g) * L::LDT + t;
            bp[j] = (which ? B1 : B0) + t * L::LDN + nt * 8 + g;
            cnt += tile < ntiles;
        }
        for (int ks = 0; ks < ksteps; ++ks) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (j < cnt) dmma(acc[j], ap[j][ks * 4], bp[j][ks * 4 * L::LDN]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (j < cnt) {
                const int tile = t0 + j * L::GW;
                const int which = tile / per, loc = tile % per;
                const int mt = loc / L::NTN, nt = loc % L::NTN;
                double* c = (which ? C1 : C0) + (mt * 8 + g) * L::LDN + nt * 8 + 2 * t;
                c[0] = acc[j][0];
                c[1] = acc[j][1];
            }
        }
    }
}

// Y[MY x NP] += A^T B where A is [K x LDT] (rows = reduction index, columns = Y rows) and B is
// [K x LDN].  Warp w of the pipeline owns Y tiles w, w + GW, ...; each tile keeps two partial accumulators (even
// and odd k-steps) and the tiles advance together, so consecutive mma never share an accumulator.
template <class L>
__device__ __forceinline__ void cta_gemm_acc_t(const double* A, const double* B, double (&y)[L::YPW][2][2], int krows,
                                               int warp, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const double* ac[L::YPW];
    const double* bc[L::YPW];
    bool on[L::YPW];
#pragma unroll
    for (int j = 0; j < L::YPW; ++j) {
        const int tile = warp + j * L::GW;
        on[j] = tile < L::YT;
        const int tt = on[j] ? tile : 0;
        const int ym = tt % L::MYT, yn = tt / L::MYT;
        ac[j] = A + t * L::LDT + ym * 8 + g;
        bc[j] = B + t * L::LDN + yn * 8 + g;
    }
    const int ks_n = krows / 4;
    int ks = 0;
    for (; ks + 1 < ks_n; ks += 2) {
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int j = 0; j < L::YPW; ++j)
                if (on[j]) dmma(y[j][h], ac[j][(ks + h) * 4 * L::LDT], bc[j][(ks + h) * 4 * L::LDN]);
    }
    if (ks < ks_n) {
#pragma unroll
        for (int j = 0; j < L::YPW; ++j)
            if (on[j]) dmma(y[j][0], ac[j][ks * 4 * L::LDT], bc[j][ks * 4 * L::LDN]);
    }
}

// Barrier over the GT threads of tile pipeline `grp` (named barrier 1 + grp; 0 is __syncthreads).
template <int GT>
__device__ __forceinline__ void mma_group_sync(int grp) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(GT) : "memory");
}

template <class S>
__global__ void __launch_bounds__(MmaTile<S>::NT, (S::D == 2) ? 2 : 1)
    apply_mma_kernel(DevOp<double> op, MmaTiles mt, const double* __restrict__ x, double* __restrict__ y, int64_t ld,
                     int nrhs) {
    using L = MmaTile<S>;
    constexpr int D = S::D, NBF = S::NBF, Q = S::Q, BS = S::BS, DD = S::DD, NF = S::NF;
    constexpr int TE = L::TE, GT = L::GT, LDN = L::LDN, LDT = L::LDT;
    const int Nq = op.Nq, nq = op.nq;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int grp = warp / L::GW, gw = warp % L::GW, gtid = tid - grp * GT;
    const MmaLayout lay = mma_layout<S>(Nq, nq);

    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sm = reinterpret_cast<double*>(smem_raw);
    double* TV = sm;
    double* TF = sm + lay.off_TF;
    double* gbuf = sm + lay.off_grp + grp * lay.grp;
    double* sU = gbuf + lay.off_U;
    double* sUN = gbuf + lay.off_UN;
    double* R0 = gbuf + lay.off_R0;
    double* R1 = gbuf + lay.off_R1;
    __shared__ int s_el_all[L::NGRP][TE];
    __shared__ int s_nb_all[L::NGRP][TE];
    int* s_el = s_el_all[grp];
    int* s_nb = s_nb_all[grp];

    for (int i = tid; i < mt.table_doubles; i += L::NT) sm[i] = mt.tables[i];
    __syncthreads();

    const int64_t nwork = static_cast<int64_t>(mt.ntiles) * nrhs;
    for (int64_t work = static_cast<int64_t>(blockIdx.x) * L::NGRP + grp; work < nwork;
         work += static_cast<int64_t>(gridDim.x) * L::NGRP) {
        int64_t t64, rhs;
        work_tile_rhs(work, mt.ntiles, nrhs, t64, rhs);
        const int tile = static_cast<int>(t64);
        const double* xr = x + rhs * ld;
        double* yr = y + rhs * ld;
        const int4 td = mt.tiles[tile];
        const int cnt = td.y, sig = td.z;
        mma_group_sync<GT>(grp);
        if (gtid < TE) s_el[gtid] = (gtid < cnt) ? mt.perm[td.x + gtid] : -1;
        mma_group_sync<GT>(grp);
        // U[k][te * Q + r]; padding rows / columns zero
        for (int i = gtid; i < L::KP * L::NP; i += GT) {
            const int k = i / L::NP, c = i % L::NP;
            const int te = c / Q, r = c % Q;
            double v = 0.0;
            if (k < NBF && c < L::NC && s_el[te] >= 0) v = xr[static_cast<int64_t>(s_el[te]) * BS + k + NBF * r];
            sU[k * LDN + c] = v;
        }
        mma_group_sync<GT>(grp);

        double yacc[L::YPW][2][2];
#pragma unroll
        for (int j = 0; j < L::YPW; ++j) yacc[j][0][0] = yacc[j][0][1] = yacc[j][1][0] = yacc[j][1][1] = 0.0;

        // ---------------- volume ----------------
        for (int q0 = 0; q0 < Nq; q0 += L::QC) {
            const int nqc = (Nq - q0 < L::QC) ? (Nq - q0) : L::QC;
            const int rows = round8(nqc * D);
            cta_gemm_store<L>(TV + q0 * D * LDT, sU, R0, rows, L::KP / 4, gw, lane);
            mma_group_sync<GT>(grp);
            for (int it = gtid; it < TE * nqc; it += GT) {
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
                        double sig[D];
#pragma unroll
                        for (int j = 0; j < D; ++j) sig[j] = mu * (Ju[uu][j] + Ju[j][uu]) + ((uu == j) ? lam * div : 0.0);
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            double s = 0.0;
#pragma unroll
                            for (int j = 0; j < D; ++j) s += G[a * D + j] * sig[j];
                            T[a][uu] = s;
                        }
                    }
#pragma unroll
                    for (int a = 0; a < D; ++a)
#pragma unroll
                        for (int uu = 0; uu < D; ++uu) rr[a * LDN + uu] = T[a][uu];
                }
            }
            mma_group_sync<GT>(grp);
            cta_gemm_acc_t<L>(TV + q0 * D * LDT, R0, yacc, rows, gw, lane);
            mma_group_sync<GT>(grp);
        }

        // ---------------- facets ----------------
#pragma unroll 1
        for (int f = 0; f < NF; ++f) {
            const int lp = (sig >> (2 * f)) & 3;
            if (gtid < TE) s_nb[gtid] = (s_el[gtid] >= 0) ? op.sides[static_cast<int64_t>(s_el[gtid]) * NF + f].z : -1;
            mma_group_sync<GT>(grp);
            for (int i = gtid; i < L::KP * L::NP; i += GT) {
                const int k = i / L::NP, c = i % L::NP;
                const int te = c / Q, r = c % Q;
                double v = 0.0;
                if (k < NBF && c < L::NC && s_nb[te] >= 0) v = xr[static_cast<int64_t>(s_nb[te]) * BS + k + NBF * r];
                sUN[k * LDN + c] = v;
            }
            mma_group_sync<GT>(grp);
            cta_gemm_store2<L>(TF + f * lay.MF * LDT, sU, R0, TF + lp * lay.MF * LDT, sUN, R1, lay.MF, L::KP / 4, gw,
                               lane);
            mma_group_sync<GT>(grp);
            for (int it = gtid; it < TE * nq; it += GT) {
                const int te = it % TE, q = it / TE;
                const int el = s_el[te];
                if (el < 0) continue;
                double* ga = R0 + (q * D) * LDN + te * Q;        // gradient rows (own) -> lift input A
                double* gb = R0 + (D * nq + q) * LDN + te * Q;   // value row (own) -> lift input B
                const double* ha = R1 + (q * D) * LDN + te * Q;
                const double* hb = R1 + (D * nq + q) * LDN + te * Q;
                const int4 sd = op.sides[static_cast<int64_t>(el) * NF + f];
                const int bcv = sd.y >> 8;
                const bool skel = sd.z != el;
                const bool fd = (bcv == 3 || bcv == 5);
                const int mode = (bcv == 0 || (skel && fd)) ? 1 : (fd ? 2 : 0);
                if (mode == 0) {
#pragma unroll
                    for (int a = 0; a < D; ++a)
#pragma unroll
                        for (int uu = 0; uu < Q; ++uu) ga[a * LDN + uu] = 0.0;
#pragma unroll
                    for (int uu = 0; uu < Q; ++uu) gb[uu] = 0.0;
                    continue;
                }
                const int fct = sd.x;
                const int side = sd.y & 0xff;
                const int own = skel ? side : 0, oth = skel ? 1 - side : 0;
                const double flip = (skel && side == 1) ? -1.0 : 1.0;
                double n[D], nu[D];
#pragma unroll
                for (int i = 0; i < D; ++i) {
                    n[i] = flip * op.fN[(static_cast<int64_t>(fct) * D + i) * nq + q];
                    nu[i] = flip * op.fNunit[(static_cast<int64_t>(fct) * D + i) * nq + q];
                }
                const double pen = op.penalty[fct];
                const double wq = op.w[q];
                double u0[Q], u1[Q], g0[D][Q], g1[D][Q];
#pragma unroll
                for (int r = 0; r < Q; ++r) {
                    u0[r] = gb[r];
                    u1[r] = (mode == 1) ? hb[r] : 0.0;
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        g0[a][r] = ga[a * LDN + r];
                        g1[a][r] = (mode == 1) ? ha[a * LDN + r] : 0.0;
                    }
                }
                if constexpr (S::KIND == kPoisson) {
                    double KG0[DD], KG1[DD];
                    const double* kg = op.fCoef + static_cast<int64_t>(fct) * 2 * DD * nq + q;
#pragma unroll
                    for (int c = 0; c < DD; ++c) {
                        KG0[c] = kg[(own * DD + c) * nq];
                        KG1[c] = kg[(oth * DD + c) * nq];
                    }
                    double uh, sg[D];
                    if (mode == 1) {
                        uh = 0.5 * (u1[0] - u0[0]);
                        const double pj = pen * (u0[0] - u1[0]);
#pragma unroll
                        for (int p = 0; p < D; ++p) {
                            double s = 0.0;
#pragma unroll
                            for (int a = 0; a < D; ++a) s += KG0[a * D + p] * g0[a][0] + KG1[a * D + p] * g1[a][0];
                            sg[p] = 0.5 * s - pj * nu[p];
                        }
                    } else {
                        uh = -u0[0];
                        const double pj = pen * u0[0];
#pragma unroll
                        for (int p = 0; p < D; ++p) {
                            double s = 0.0;
#pragma unroll
                            for (int a = 0; a < D; ++a) s += KG0[a * D + p] * g0[a][0];
                            sg[p] = s - pj * nu[p];
                        }
                    }
                    double bsum = 0.0;
#pragma unroll
                    for (int r = 0; r < D; ++r) bsum += n[r] * sg[r];
                    gb[0] = -wq * bsum;
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        double s = 0.0;
#pragma unroll
                        for (int r = 0; r < D; ++r) s += n[r] * KG0[a * D + r];
                        ga[a * LDN] = wq * uh * s;
                    }
                } else {
                    double G0[DD], G1[DD];
                    const double* gg = op.fG + static_cast<int64_t>(fct) * 2 * DD * nq + q;
#pragma unroll
                    for (int c = 0; c < DD; ++c) {
                        G0[c] = gg[(own * DD + c) * nq];
                        G1[c] = gg[(oth * DD + c) * nq];
                    }
                    const double* lm = op.fCoef + static_cast<int64_t>(fct) * 4 * nq + q;
                    const double lam0 = lm[(2 * own + 0) * nq], mu0 = lm[(2 * own + 1) * nq];
                    const double lam1 = lm[(2 * oth + 0) * nq], mu1 = lm[(2 * oth + 1) * nq];
                    double sg[D][D];
                    {
                        double J0[D][D];
#pragma unroll
                        for (int s = 0; s < D; ++s)
#pragma unroll
                            for (int r = 0; r < D; ++r) {
                                double acc0 = 0.0;
#pragma unroll
                                for (int a = 0; a < D; ++a) acc0 += G0[a * D + s] * g0[a][r];
                                J0[s][r] = acc0;
                            }
                        double d0 = 0.0;
#pragma unroll
                        for (int r = 0; r < D; ++r) d0 += J0[r][r];
#pragma unroll
                        for (int i = 0; i < D; ++i)
#pragma unroll
                            for (int j = 0; j < D; ++j) sg[i][j] = mu0 * (J0[i][j] + J0[j][i]) + ((i == j) ? lam0 * d0 : 0.0);
                    }
                    double uhm[D];
                    if (mode == 1) {
                        double J1[D][D];
#pragma unroll
                        for (int s = 0; s < D; ++s)
#pragma unroll
                            for (int r = 0; r < D; ++r) {
                                double acc1 = 0.0;
#pragma unroll
                                for (int a = 0; a < D; ++a) acc1 += G1[a * D + s] * g1[a][r];
                                J1[s][r] = acc1;
                            }
                        double d1 = 0.0;
#pragma unroll
                        for (int r = 0; r < D; ++r) d1 += J1[r][r];
#pragma unroll
                        for (int i = 0; i < D; ++i) {
                            const double pj = pen * (u0[i] - u1[i]);
#pragma unroll
                            for (int j = 0; j < D; ++j) {
                                const double s1 = mu1 * (J1[i][j] + J1[j][i]) + ((i == j) ? lam1 * d1 : 0.0);
                                sg[i][j] = 0.5 * (sg[i][j] + s1) - pj * nu[j];
                            }
                            uhm[i] = 0.5 * (u1[i] - u0[i]);
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < D; ++i) {
                            const double pj = pen * u0[i];
#pragma unroll
                            for (int j = 0; j < D; ++j) sg[i][j] -= pj * nu[j];
                            uhm[i] = -u0[i];
                        }
                    }
                    double un = 0.0;
#pragma unroll
                    for (int r = 0; r < D; ++r) un += uhm[r] * n[r];
#pragma unroll
                    for (int uu = 0; uu < D; ++uu) {
                        double X[D];
#pragma unroll
                        for (int j = 0; j < D; ++j)
                            X[j] = mu0 * (uhm[uu] * n[j] + uhm[j] * n[uu]) + ((uu == j) ? lam0 * un : 0.0);
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            double s = 0.0;
#pragma unroll
                            for (int j = 0; j < D; ++j) s += G0[a * D + j] * X[j];
                            ga[a * LDN + uu] = wq * s;
                        }
                        double bsum = 0.0;
#pragma unroll
                        for (int j = 0; j < D; ++j) bsum += n[j] * sg[uu][j];
                        gb[uu] = -wq * bsum;
                    }
                }
            }
            mma_group_sync<GT>(grp);
            cta_gemm_acc_t<L>(TF + f * lay.MF * LDT, R0, yacc, lay.MF, gw, lane);
            mma_group_sync<GT>(grp);
        }

        // ---------------- write the output tile ----------------
        {
            const int g = lane >> 2, t = lane & 3;
#pragma unroll
            for (int j = 0; j < L::YPW; ++j) {
                const int tl = gw + j * L::GW;
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
}

}  // namespace tdg
