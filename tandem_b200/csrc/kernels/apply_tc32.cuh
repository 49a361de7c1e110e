// FP32 operator apply on the tensor cores: mma.sync m16n8k8 with TF32 operands in the split
// ("3xTF32") form a*b ~ a_hi*b_hi + a_hi*b_lo + a_lo*b_hi, where a_hi = tf32(a) and
// a_lo = tf32(a - a_hi).  Each product then carries about 21 significant bits, close to FP32,
// and every sum is accumulated in FP32.  This is the inner operator of the mixed-precision solve
// (FP32 Krylov iterations inside FP64 iterative refinement); the facet penalty products are formed
// in FP64 and rounded once.
//
// Same algorithm and data flow as the FP64 kernel of apply_mma.cuh (tandem's element-centric
// apply: volume term, then per local face the own/neighbour traces, the numerical fluxes and the
// lift-back; see apply.cuh for the reference citations), with a different work split:
//
//   * a tile holds TE elements; its columns are (element, component) pairs, c = te * Q + r;
//   * forward GEMMs R = T x U (T: basis table in shared memory, U: the tile's coefficients) are
//     cut into units (16-row m-tile, group of NPW 8-column n-tiles), so every table fragment a
//     warp loads and splits feeds 3 * NPW mma;
//   * back-projections Y += T^T R accumulate in registers for the whole tile.  The Y units
//     (16-row m-tile of Y, n-tile group) are owned by fixed warps; when there are fewer units than
//     warps, KSP warps share a unit and split the reduction index, and the partial sums meet in
//     shared memory once per tile, where the output block is also staged for coalesced stores.
//
//   * the CTA runs NGRP independent tile pipelines ("groups" of GW warps with their own buffers and
//     named barriers) that share the resident tables, so one group's global-memory waits overlap
//     the other group's tensor work.
//
// Shared-memory strides: tables and U use ld = 4 (mod 8) floats (conflict-free A / B fragment
// loads of the forward GEMM); R uses ld = 8 or 24 (mod 32) floats (conflict-free C stores and B
// loads of the back-projection).  The transposed table reads of the back-projection have 2-way
// conflicts.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace tdg {

__host__ __device__ constexpr int tc_round(int x, int m) { return (x + m - 1) / m * m; }
__host__ __device__ constexpr int tc_ldr(int np) {
    return (np % 32 == 8 || np % 32 == 24) ? np : tc_ldr(np + 8);
}

// Elements per tile: 48 columns for 3D elasticity, 64 otherwise.
__host__ __device__ constexpr int tc32_tile_elements(int D, int Q) { return ((D == 3 && Q == 3) ? 48 : 64) / Q; }

__host__ __device__ constexpr int tc_npw(int ntn) {
    return (ntn % 6 == 0) ? 6 : ((ntn % 4 == 0) ? 4 : ((ntn % 3 == 0) ? 3 : ((ntn % 2 == 0) ? 2 : 1)));
}

template <class S>
struct Tc32Tile {
    static constexpr int TE = tc32_tile_elements(S::D, S::Q);
    static constexpr int NC = TE * S::Q;
    static constexpr int NP = tc_round(NC, 8);
    static constexpr int NTN = NP / 8;
    static constexpr int NPW = tc_npw(NTN);                        // n-tiles per unit
    static constexpr int NG = NTN / NPW;
    static constexpr int KP = tc_round(S::NBF, 8);
    static constexpr int KS = KP / 8;
    static constexpr int LDT = KP + 4;  // = 4 mod 8
    static constexpr int LDU = LDT;
    static constexpr int LDR = tc_ldr(NP);
    static constexpr int MY = tc_round(S::NBF, 16);
    static constexpr int MYT = MY / 16;
    static constexpr int YU = MYT * NG;                            // Y units per tile
    static constexpr int NGRP = (S::D == 3) ? 2 : 1;               // tile pipelines per CTA
    static constexpr int GW = (S::D == 3) ? 6 : 8;                 // warps per pipeline
    static constexpr int GT = 32 * GW;
    static constexpr int NW = GW * NGRP;
    static constexpr int NT = 32 * NW;
    static constexpr int KSP = (YU >= GW) ? 1 : GW / YU;
    static constexpr int UPW = (YU + GW - 1) / GW;
    static constexpr int QCP = (S::D == 3) ? 32 : 64;              // volume points per chunk
    static constexpr int MINB = (S::D == 2) ? 2 : 1;
};

struct Tc32Layout {
    int MV, MF;                 // padded rows of TV and of each TF (multiples of 16)
    int off_TF;                 // tables: TV at 0, TF at off_TF
    int off_grp, grp;           // first pipeline buffer and the floats of one pipeline's buffers
    int off_U, off_UN, off_R0, off_R1;  // offsets inside a pipeline's buffers
    int total;                  // floats
};

template <class S>
__host__ __device__ inline Tc32Layout tc32_layout(int Nq, int nq) {
    using L = Tc32Tile<S>;
    Tc32Layout l;
    l.MV = tc_round(S::D * Nq, 16);
    l.MF = tc_round((S::D + 1) * nq, 16);
    int vrows = tc_round(S::D * L::QCP, 16);
    if (vrows > l.MV) vrows = l.MV;
    const int r0_rows = vrows > l.MF ? vrows : l.MF;
    int r0 = r0_rows * L::LDR;
    const int stage = L::KSP * L::NP * L::MY;  // Y partials / output staging
    if (stage > r0) r0 = stage;
    l.off_TF = l.MV * L::LDT;
    l.off_grp = l.off_TF + S::NF * l.MF * L::LDT;
    l.off_U = 0;
    l.off_UN = l.off_U + L::NP * L::LDU;
    l.off_R0 = l.off_UN + L::NP * L::LDU;
    l.off_R1 = l.off_R0 + r0;
    l.grp = l.off_R1 + l.MF * L::LDR;
    l.total = l.off_grp + L::NGRP * l.grp;
    return l;
}

struct Tc32Tiles {
    const int4* tiles = nullptr;   // {first index into perm, count, signature, 0}
    const int* perm = nullptr;     // element ids grouped by neighbour-face signature
    const float* tables = nullptr; // TV then TF[0..NF-1], packed as in shared memory
    int ntiles = 0;
    int table_floats = 0;
    int* status = nullptr;         // device word: non-zero once a bounded wait of the tcgen05 kernel ran out
};

// x = hi + lo with hi = x rounded to TF32 (nearest, ties away from zero: add half an ulp of the
// 10-bit mantissa to the magnitude bits, then clear the 13 low bits).  lo is passed as is: the
// tensor core reads the upper 19 bits of a TF32 operand, so lo loses at most 2^-11 of itself,
// i.e. 2^-22 of x.
__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo) {
    const uint32_t h = (__float_as_uint(x) + 0x1000u) & 0xffffe000u;
    hi = h;
    lo = __float_as_uint(x - __uint_as_float(h));
}

// Barrier over the GT threads of pipeline `grp` (named barrier 1 + grp; 0 is __syncthreads).
template <int GT>
__device__ __forceinline__ void group_sync(int grp) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(GT) : "memory");
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// a += x*y in the 3xTF32 form (small terms first); NP = 1: one TF32 pass (hi hi, about 2^-11 per
// product), for preconditioner applies.
template <int NP = 3>
__device__ __forceinline__ void mma3(float (&c)[4], const uint32_t (&ah)[4], const uint32_t (&al)[4], uint32_t bh0,
                                     uint32_t bh1, uint32_t bl0, uint32_t bl1) {
    if constexpr (NP == 3) {
        mma_tf32(c, al, bh0, bh1);
        mma_tf32(c, ah, bl0, bl1);
    }
    mma_tf32(c, ah, bh0, bh1);
}

// The same for NPW accumulators sharing one A fragment, the three products of each accumulator in
// the same order but interleaved across the accumulators, so that consecutive mma are independent
// (three dependent mma per accumulator would otherwise stall on each other's latency).
template <int NPW, int NP = 3>
__device__ __forceinline__ void mma3_rows(float (&c)[NPW][4], const uint32_t (&ah)[4], const uint32_t (&al)[4],
                                          const uint32_t (&bh0)[NPW], const uint32_t (&bh1)[NPW],
                                          const uint32_t (&bl0)[NPW], const uint32_t (&bl1)[NPW]) {
    if constexpr (NP == 3) {
#pragma unroll
        for (int j = 0; j < NPW; ++j) mma_tf32(c[j], al, bh0[j], bh1[j]);
#pragma unroll
        for (int j = 0; j < NPW; ++j) mma_tf32(c[j], ah, bl0[j], bl1[j]);
    }
#pragma unroll
    for (int j = 0; j < NPW; ++j) mma_tf32(c[j], ah, bh0[j], bh1[j]);
}
// 3xTF32 products interleaved across a row's accumulators (mma3_rows) or one accumulator at a time.
constexpr bool kMma3Interleave = true;

// Forward GEMMs: for each of `nops` (1 or 2) operand pairs (A_i: table rows [mtiles*16][LDT], B_i: U
// [NP][LDU] column-major), R_i[m][c] = sum_k A_i[m][k] B_i[c][k], stored with ld LDR.  Units
// (operand, m-tile, n-group) are dealt round-robin to the warps of the pipeline; each table
// fragment a warp loads (and splits) feeds the NPW n-tiles of its unit.
template <class L, int NP = 3>
__device__ __forceinline__ void tc_forward(const float* A0, const float* B0, float* R0, const float* A1, const float* B1,
                                           float* R1, int nops, int mtiles, int warp, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int per_op = mtiles * L::NG;
    const int units = nops * per_op;
    for (int u = warp; u < units; u += L::GW) {
        const int op = u / per_op, rem = u % per_op;
        const int ng = rem / mtiles, mt = rem % mtiles;
        const float* bp = (op ? B1 : B0) + (ng * L::NPW * 8 + g) * L::LDU + t;
        float acc[L::NPW][4];
#pragma unroll
        for (int j = 0; j < L::NPW; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
        const float* ap = (op ? A1 : A0) + (mt * 16 + g) * L::LDT + t;
#pragma unroll
        for (int ks = 0; ks < L::KS; ++ks) {
            uint32_t ah[4], al[4];
            tf32_split(ap[ks * 8], ah[0], al[0]);
            tf32_split(ap[ks * 8 + 8 * L::LDT], ah[1], al[1]);
            tf32_split(ap[ks * 8 + 4], ah[2], al[2]);
            tf32_split(ap[ks * 8 + 4 + 8 * L::LDT], ah[3], al[3]);
            if constexpr (kMma3Interleave) {
                uint32_t bh0[L::NPW], bl0[L::NPW], bh1[L::NPW], bl1[L::NPW];
#pragma unroll
                for (int j = 0; j < L::NPW; ++j) {
                    tf32_split(bp[j * 8 * L::LDU + ks * 8], bh0[j], bl0[j]);
                    tf32_split(bp[j * 8 * L::LDU + ks * 8 + 4], bh1[j], bl1[j]);
                }
                mma3_rows<L::NPW, NP>(acc, ah, al, bh0, bh1, bl0, bl1);
            } else {
#pragma unroll
                for (int j = 0; j < L::NPW; ++j) {
                    uint32_t bh0, bl0, bh1, bl1;
                    tf32_split(bp[j * 8 * L::LDU + ks * 8], bh0, bl0);
                    tf32_split(bp[j * 8 * L::LDU + ks * 8 + 4], bh1, bl1);
                    mma3<NP>(acc[j], ah, al, bh0, bh1, bl0, bl1);
                }
            }
        }
        float* rp = (op ? R1 : R0) + (mt * 16 + g) * L::LDR + ng * L::NPW * 8 + 2 * t;
#pragma unroll
        for (int j = 0; j < L::NPW; ++j) {
            *reinterpret_cast<float2*>(rp + j * 8) = make_float2(acc[j][0], acc[j][1]);
            *reinterpret_cast<float2*>(rp + j * 8 + 8 * L::LDR) = make_float2(acc[j][2], acc[j][3]);
        }
    }
}

// Back-projection Y += A^T R over `mrows` reduction rows (a multiple of 8): A is a table
// [mrows][LDT] (Y row index = table column), R is [mrows][LDR].  Warp w owns Y units
// w % YU (+ NW, ...) for reduction part w / YU (k-steps kp, kp + KSP, ...).
template <class L, int NP = 3>
__device__ __forceinline__ void tc_backproject(const float* A, const float* R, float (&y)[L::UPW][L::NPW][4], int mrows,
                                               int warp, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int kp = warp / L::YU;
    if (kp >= L::KSP) return;
    const int ksteps = mrows / 8;
#pragma unroll
    for (int uu = 0; uu < L::UPW; ++uu) {
        const int unit = (warp % L::YU) + uu * L::GW;
        if (L::UPW > 1 && unit >= L::YU) break;
        const int myt = unit % L::MYT, ng = unit / L::MYT;
        const float* ap = A + t * L::LDT + myt * 16 + g;
        const float* rp = R + t * L::LDR + ng * L::NPW * 8 + g;
        for (int ks = kp; ks < ksteps; ks += L::KSP) {
            uint32_t ah[4], al[4];
            const float* a = ap + ks * 8 * L::LDT;
            tf32_split(a[0], ah[0], al[0]);
            tf32_split(a[8], ah[1], al[1]);
            tf32_split(a[4 * L::LDT], ah[2], al[2]);
            tf32_split(a[4 * L::LDT + 8], ah[3], al[3]);
            const float* r = rp + ks * 8 * L::LDR;
            if constexpr (kMma3Interleave) {
                uint32_t bh0[L::NPW], bl0[L::NPW], bh1[L::NPW], bl1[L::NPW];
#pragma unroll
                for (int j = 0; j < L::NPW; ++j) {
                    tf32_split(r[j * 8], bh0[j], bl0[j]);
                    tf32_split(r[j * 8 + 4 * L::LDR], bh1[j], bl1[j]);
                }
                mma3_rows<L::NPW, NP>(y[uu], ah, al, bh0, bh1, bl0, bl1);
            } else {
#pragma unroll
                for (int j = 0; j < L::NPW; ++j) {
                    uint32_t bh0, bl0, bh1, bl1;
                    tf32_split(r[j * 8], bh0, bl0);
                    tf32_split(r[j * 8 + 4 * L::LDR], bh1, bl1);
                    mma3<NP>(y[uu][j], ah, al, bh0, bh1, bl0, bl1);
                }
            }
        }
    }
}

// TX: the vectors' type -- float, or double for the mixed solve (FP32 operator arithmetic on FP64
// vectors: x is rounded to FP32 when it is gathered, y widened when it is stored).
template <class S, typename TX, int NP = 3>
__global__ void __launch_bounds__(Tc32Tile<S>::NT, Tc32Tile<S>::MINB)
    apply_tc32_kernel(DevOp<float> op, Tc32Tiles mt, const TX* __restrict__ x, TX* __restrict__ y, int64_t ld,
                      int nrhs) {
    using L = Tc32Tile<S>;
    constexpr int D = S::D, NBF = S::NBF, Q = S::Q, BS = S::BS, DD = S::DD, NF = S::NF;
    constexpr int TE = L::TE, GT = L::GT, LDR = L::LDR, LDT = L::LDT, LDU = L::LDU;
    const int Nq = op.Nq, nq = op.nq;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int grp = warp / L::GW, gw = warp % L::GW, gtid = tid - grp * GT;
    const Tc32Layout lay = tc32_layout<S>(Nq, nq);

    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* sm = reinterpret_cast<float*>(smem_raw);
    float* TV = sm;
    float* TF = sm + lay.off_TF;
    float* gbuf = sm + lay.off_grp + grp * lay.grp;
    float* sU = gbuf + lay.off_U;
    float* sUN = gbuf + lay.off_UN;
    float* R0 = gbuf + lay.off_R0;
    float* R1 = gbuf + lay.off_R1;
    __shared__ int s_el_all[L::NGRP][TE];
    __shared__ int s_nb_all[L::NGRP][TE];
    int* s_el = s_el_all[grp];
    int* s_nb = s_nb_all[grp];

    for (int i = tid; i < mt.table_floats; i += L::NT) sm[i] = mt.tables[i];
    __syncthreads();

    const int64_t nwork = static_cast<int64_t>(mt.ntiles) * nrhs;
    for (int64_t work = static_cast<int64_t>(blockIdx.x) * L::NGRP + grp; work < nwork;
         work += static_cast<int64_t>(gridDim.x) * L::NGRP) {
        int64_t t64, rhs;
        work_tile_rhs(work, mt.ntiles, nrhs, t64, rhs);
        const int tile = static_cast<int>(t64);
        const TX* xr = x + rhs * ld;
        TX* yr = y + rhs * ld;
        const int4 td = mt.tiles[tile];
        const int cnt = td.y, sig = td.z;
        group_sync<GT>(grp);
        if (gtid < TE) s_el[gtid] = (gtid < cnt) ? mt.perm[td.x + gtid] : -1;
        group_sync<GT>(grp);
        // U[c][k] (column-major); padding zero
        for (int i = gtid; i < L::NP * L::KP; i += GT) {
            const int c = i / L::KP, k = i % L::KP;
            const int te = c / Q, r = c % Q;
            float v = 0.0f;
            if (k < NBF && c < L::NC && s_el[te] >= 0)
                v = static_cast<float>(xr[static_cast<int64_t>(s_el[te]) * BS + k + NBF * r]);
            sU[c * LDU + k] = v;
        }
        group_sync<GT>(grp);

        float yacc[L::UPW][L::NPW][4];
#pragma unroll
        for (int a = 0; a < L::UPW; ++a)
#pragma unroll
            for (int j = 0; j < L::NPW; ++j) yacc[a][j][0] = yacc[a][j][1] = yacc[a][j][2] = yacc[a][j][3] = 0.0f;

        // ---------------- volume, in chunks of QCP points ----------------
        for (int q0 = 0; q0 < Nq; q0 += L::QCP) {
            const int nqc = (Nq - q0 < L::QCP) ? (Nq - q0) : L::QCP;
            const int rows = tc_round(nqc * D, 16);
            if (q0 > 0) group_sync<GT>(grp);  // previous chunk's back-projection done with R0
            tc_forward<L, NP>(TV + q0 * D * LDT, sU, R0, TV, sU, R0, 1, rows / 16, gw, lane);
            group_sync<GT>(grp);
            for (int it = gtid; it < TE * nqc; it += GT) {
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
            group_sync<GT>(grp);
            tc_backproject<L, NP>(TV + q0 * D * LDT, R0, yacc, rows, gw, lane);
        }

        // ---------------- facets ----------------
#pragma unroll 1
        for (int f = 0; f < NF; ++f) {
            const int lp = (sig >> (2 * f)) & 3;
            group_sync<GT>(grp);  // previous back-projection done with R0 / sUN
            if (gtid < TE) s_nb[gtid] = (s_el[gtid] >= 0) ? op.sides[static_cast<int64_t>(s_el[gtid]) * NF + f].z : -1;
            group_sync<GT>(grp);
            for (int i = gtid; i < L::NP * L::KP; i += GT) {
                const int c = i / L::KP, k = i % L::KP;
                const int te = c / Q, r = c % Q;
                float v = 0.0f;
                if (k < NBF && c < L::NC && s_nb[te] >= 0)
                    v = static_cast<float>(xr[static_cast<int64_t>(s_nb[te]) * BS + k + NBF * r]);
                sUN[c * LDU + k] = v;
            }
            group_sync<GT>(grp);
            tc_forward<L, NP>(TF + f * lay.MF * LDT, sU, R0, TF + lp * lay.MF * LDT, sUN, R1, 2, lay.MF / 16, gw, lane);
            group_sync<GT>(grp);
            for (int it = gtid; it < TE * nq; it += GT) {
                const int te = it % TE, q = it / TE;
                const int el = s_el[te];
                if (el < 0) continue;
                float* ga = R0 + (q * D) * LDR + te * Q;
                float* gb = R0 + (D * nq + q) * LDR + te * Q;
                const float* ha = R1 + (q * D) * LDR + te * Q;
                const float* hb = R1 + (D * nq + q) * LDR + te * Q;
                const int4 sd = op.sides[static_cast<int64_t>(el) * NF + f];
                const int bcv = sd.y >> 8;
                const bool skel = sd.z != el;
                const bool fd = (bcv == 3 || bcv == 5);
                const int mode = (bcv == 0 || (skel && fd)) ? 1 : (fd ? 2 : 0);
                if (mode == 0) {
#pragma unroll
                    for (int a = 0; a < D; ++a)
#pragma unroll
                        for (int uu = 0; uu < Q; ++uu) ga[a * LDR + uu] = 0.0f;
#pragma unroll
                    for (int uu = 0; uu < Q; ++uu) gb[uu] = 0.0f;
                    continue;
                }
                const int fct = sd.x;
                const int side = sd.y & 0xff;
                const int own = skel ? side : 0, oth = skel ? 1 - side : 0;
                const float flip = (skel && side == 1) ? -1.0f : 1.0f;
                float n[D], nu[D];
#pragma unroll
                for (int i = 0; i < D; ++i) {
                    n[i] = flip * op.fN[(static_cast<int64_t>(fct) * D + i) * nq + q];
                    nu[i] = flip * op.fNunit[(static_cast<int64_t>(fct) * D + i) * nq + q];
                }
                const double pen = op.penalty[fct];
                const float wq = op.w[q];
                float u0[Q], u1[Q], g0[D][Q], g1[D][Q];
#pragma unroll
                for (int r = 0; r < Q; ++r) {
                    u0[r] = gb[r];
                    u1[r] = (mode == 1) ? hb[r] : 0.0f;
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        g0[a][r] = ga[a * LDR + r];
                        g1[a][r] = (mode == 1) ? ha[a * LDR + r] : 0.0f;
                    }
                }
                if constexpr (S::KIND == kPoisson) {
                    float KG0[DD], KG1[DD];
                    const float* kg = op.fCoef + static_cast<int64_t>(fct) * 2 * DD * nq + q;
#pragma unroll
                    for (int c = 0; c < DD; ++c) {
                        KG0[c] = kg[(own * DD + c) * nq];
                        KG1[c] = kg[(oth * DD + c) * nq];
                    }
                    float uh, sg[D];
                    if (mode == 1) {
                        uh = 0.5f * (u1[0] - u0[0]);
                        const float pj = static_cast<float>(pen * (static_cast<double>(u0[0]) - u1[0]));
#pragma unroll
                        for (int p = 0; p < D; ++p) {
                            float s = 0.0f;
#pragma unroll
                            for (int a = 0; a < D; ++a) s += KG0[a * D + p] * g0[a][0] + KG1[a * D + p] * g1[a][0];
                            sg[p] = 0.5f * s - pj * nu[p];
                        }
                    } else {
                        uh = -u0[0];
                        const float pj = static_cast<float>(pen * u0[0]);
#pragma unroll
                        for (int p = 0; p < D; ++p) {
                            float s = 0.0f;
#pragma unroll
                            for (int a = 0; a < D; ++a) s += KG0[a * D + p] * g0[a][0];
                            sg[p] = s - pj * nu[p];
                        }
                    }
                    float bsum = 0.0f;
#pragma unroll
                    for (int r = 0; r < D; ++r) bsum += n[r] * sg[r];
                    gb[0] = -wq * bsum;
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        float s = 0.0f;
#pragma unroll
                        for (int r = 0; r < D; ++r) s += n[r] * KG0[a * D + r];
                        ga[a * LDR] = wq * uh * s;
                    }
                } else {
                    float G0[DD], G1[DD];
                    const float* gg = op.fG + static_cast<int64_t>(fct) * 2 * DD * nq + q;
#pragma unroll
                    for (int c = 0; c < DD; ++c) {
                        G0[c] = gg[(own * DD + c) * nq];
                        G1[c] = gg[(oth * DD + c) * nq];
                    }
                    const float* lm = op.fCoef + static_cast<int64_t>(fct) * 4 * nq + q;
                    const float lam0 = lm[(2 * own + 0) * nq], mu0 = lm[(2 * own + 1) * nq];
                    const float lam1 = lm[(2 * oth + 0) * nq], mu1 = lm[(2 * oth + 1) * nq];
                    float sg[D][D];
                    {
                        float J0[D][D];
#pragma unroll
                        for (int s = 0; s < D; ++s)
#pragma unroll
                            for (int r = 0; r < D; ++r) {
                                float acc0 = 0.0f;
#pragma unroll
                                for (int a = 0; a < D; ++a) acc0 += G0[a * D + s] * g0[a][r];
                                J0[s][r] = acc0;
                            }
                        float d0 = 0.0f;
#pragma unroll
                        for (int r = 0; r < D; ++r) d0 += J0[r][r];
#pragma unroll
                        for (int i = 0; i < D; ++i)
#pragma unroll
                            for (int j = 0; j < D; ++j) sg[i][j] = mu0 * (J0[i][j] + J0[j][i]) + ((i == j) ? lam0 * d0 : 0.0f);
                    }
                    float uhm[D];
                    if (mode == 1) {
                        float J1[D][D];
#pragma unroll
                        for (int s = 0; s < D; ++s)
#pragma unroll
                            for (int r = 0; r < D; ++r) {
                                float acc1 = 0.0f;
#pragma unroll
                                for (int a = 0; a < D; ++a) acc1 += G1[a * D + s] * g1[a][r];
                                J1[s][r] = acc1;
                            }
                        float d1 = 0.0f;
#pragma unroll
                        for (int r = 0; r < D; ++r) d1 += J1[r][r];
#pragma unroll
                        for (int i = 0; i < D; ++i) {
                            const float pj = static_cast<float>(pen * (static_cast<double>(u0[i]) - u1[i]));
#pragma unroll
                            for (int j = 0; j < D; ++j) {
                                const float s1 = mu1 * (J1[i][j] + J1[j][i]) + ((i == j) ? lam1 * d1 : 0.0f);
                                sg[i][j] = 0.5f * (sg[i][j] + s1) - pj * nu[j];
                            }
                            uhm[i] = 0.5f * (u1[i] - u0[i]);
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < D; ++i) {
                            const float pj = static_cast<float>(pen * u0[i]);
#pragma unroll
                            for (int j = 0; j < D; ++j) sg[i][j] -= pj * nu[j];
                            uhm[i] = -u0[i];
                        }
                    }
                    float un = 0.0f;
#pragma unroll
                    for (int r = 0; r < D; ++r) un += uhm[r] * n[r];
#pragma unroll
                    for (int uu = 0; uu < D; ++uu) {
                        float X[D];
#pragma unroll
                        for (int j = 0; j < D; ++j)
                            X[j] = mu0 * (uhm[uu] * n[j] + uhm[j] * n[uu]) + ((uu == j) ? lam0 * un : 0.0f);
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            float s = 0.0f;
#pragma unroll
                            for (int j = 0; j < D; ++j) s += G0[a * D + j] * X[j];
                            ga[a * LDR + uu] = wq * s;
                        }
                        float bsum = 0.0f;
#pragma unroll
                        for (int j = 0; j < D; ++j) bsum += n[j] * sg[uu][j];
                        gb[uu] = -wq * bsum;
                    }
                }
            }
            group_sync<GT>(grp);
            tc_backproject<L, NP>(TF + f * lay.MF * LDT, R0, yacc, lay.MF, gw, lane);
        }

        // ---------------- reduce the k-split partials and write the tile ----------------
        group_sync<GT>(grp);
        {
            const int g = lane >> 2, t = lane & 3;
            const int kp = gw / L::YU;
            if (kp < L::KSP) {
                float* st = R0 + kp * L::NP * L::MY;
#pragma unroll
                for (int uu = 0; uu < L::UPW; ++uu) {
                    const int unit = (gw % L::YU) + uu * L::GW;
                    if (unit >= L::YU) break;
                    const int myt = unit % L::MYT, ng = unit / L::MYT;
#pragma unroll
                    for (int j = 0; j < L::NPW; ++j) {
                        const int c = (ng * L::NPW + j) * 8 + 2 * t;
                        const int k = myt * 16 + g;
                        st[c * L::MY + k] = yacc[uu][j][0];
                        st[(c + 1) * L::MY + k] = yacc[uu][j][1];
                        st[c * L::MY + k + 8] = yacc[uu][j][2];
                        st[(c + 1) * L::MY + k + 8] = yacc[uu][j][3];
                    }
                }
            }
        }
        group_sync<GT>(grp);
        for (int i = gtid; i < L::NC * NBF; i += GT) {
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

}  // namespace tdg
