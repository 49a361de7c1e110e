// Volume term of the face-centric FP32 apply on the 5th-generation tensor cores (tcgen05.mma
// kind::tf32, accumulators in tensor memory), 3xTF32 (hi hi + hi lo + lo hi, ~2^-21 per product,
// FP32 accumulation).  It replaces vol_tc32_kernel (mma.sync) in front of face_tc32_kernel: per tile
// of TE = 16 consecutive elements it stores y = volume term (Poisson.cpp:551-575,
// Elasticity.cpp:698-745, the same contraction and pointwise flux as the FP64 kernels).
//
// Per tile (one CTA per SM, 256 threads, one tile at a time):
//  1. U: the tile's coefficient blocks, columns n = r TE + te (component-major), K = basis padded to
//     KF, split hi / lo into the core-matrix layout (K-major, tc05.cuh);
//  2. forward: for each derivative direction a, R_a[q][n] = sum_k D_a[q][k] U[n][k] into TMEM
//     (M = 128 lanes = quadrature points q < Nq <= 64, N = Q TE columns at a * NCOL);
//  3. pointwise: the warps that own lanes 0..63 (warps 0, 1, 4, 5: lane q, half of the tile's
//     elements each) read R_a[q][(r, te)] with 32x32b loads, form the stress / flux with the point's
//     J^-1 and coefficients (read coalesced over q from [E][field][Nq]) and write S[(r, te)][(a, q)]
//     split hi / lo;
//  4. backward: Y[k][n] = sum_(a, q) D_a[q][k] S[n][(a, q)] into TMEM (M = 128 lanes = basis k,
//     K = D * 64);
//  5. y: lanes k < NBF store y[e BS + k + NBF r] (32 consecutive k per warp store).
//
// Every operand is K-major in core matrices (tc05.cuh).  The table D_a[q][k] is held twice per CTA
// (hi and lo each): [k/4][a][q/8][8 q][4 k] for the forward MMA (rows q: SBO 128 bytes, K chunks:
// LBO D KB) and [(a, q)/4][k/8][8 k][4 (a, q)] for the backward one.  S's K chunks are 16 bytes
// further apart than its rows need, so that the pointwise phase's stores (32 consecutive q of one
// column per warp) fall on 32 distinct banks.  Rows of an M = 128 operand past the stored ones read
// the following shared memory; they only produce accumulator rows that are never read, and the
// buffer extends past every such read.
#pragma once

#include "apply_face.cuh"
#include "tc05.cuh"

namespace tdg {

template <class S>
struct Tc05Vol {
    static constexpr int D = S::D, Q = S::Q, NBF = S::NBF;
    static constexpr int TE = 16;                    // elements per tile
    static constexpr int NCOL = Q * TE;              // forward N, backward N: (r, te)
    static constexpr int KF = (NBF + 7) / 8 * 8;     // basis padded to the K step
    static constexpr int KC = KF / 4;                // 16-byte K chunks of the forward operands
    static constexpr int NQ = 64;                    // quadrature points per direction block
    static constexpr int KB = D * NQ;                // backward K: (a, q)
    static constexpr int NT = 256;
    static constexpr int KCS = D * NQ * 16;          // bytes between K chunks of the forward table
    static constexpr int TAB = KC * KCS;             // bytes of one forward table copy
    static constexpr int LBO_B = (KF / 8) * 128;     // bytes between K chunks of the backward table
    static constexpr int TABB = (KB / 4) * LBO_B;    // bytes of one backward table copy
    static constexpr int UB = NCOL * KF * 4;         // bytes of one U copy
    static constexpr int SCS = (NCOL / 8) * 128 + 16;  // bytes between K chunks of S (padded)
    static constexpr int SB = (KB / 4) * SCS;        // bytes of one S copy
    static constexpr int OFF_AFL = TAB, OFF_ABH = 2 * TAB, OFF_ABL = OFF_ABH + TABB, OFF_UH = OFF_ABL + TABB,
                         OFF_UL = OFF_UH + UB, OFF_SH = OFF_UL + UB, OFF_SL = OFF_SH + SB, END = OFF_SL + SB;
    // + reads of M = 128 operands past their stored rows (at most 16 row groups past a chunk),
    // + alignment of the base
    static constexpr int BYTES = END + 2048 + 1024;
    static constexpr int COLS_USED = (D + 1) * NCOL;
    static constexpr int TCOLS = COLS_USED <= 32 ? 32 : COLS_USED <= 64 ? 64 : COLS_USED <= 128 ? 128 : 256;
    static_assert(NCOL % 16 == 0 && NCOL <= 256, "M = 128 MMAs need N a multiple of 16");
    static_assert(COLS_USED <= 256, "tensor memory");
};

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float (&v)[4]) {
    uint32_t r0, r1, r2, r3;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(taddr));
    v[0] = __uint_as_float(r0);
    v[1] = __uint_as_float(r1);
    v[2] = __uint_as_float(r2);
    v[3] = __uint_as_float(r3);
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// Pointwise volume flux at one point of one element (the same arithmetic as vol_tc32_kernel):
// g[a][r] = d u_r / d xi_a in, T[a][r] (the lifted flux) out.
template <class S>
__device__ __forceinline__ void vol_point(const float (&G)[S::DD], float c0, float c1, const float (&g)[S::D][S::Q],
                                          float (&T)[S::D][S::Q]) {
    constexpr int D = S::D;
    if constexpr (S::KIND == kPoisson) {
        float gx[D];
#pragma unroll
        for (int i = 0; i < D; ++i) {
            float s = 0.0f;
#pragma unroll
            for (int a = 0; a < D; ++a) s += G[a * D + i] * g[a][0];
            gx[i] = c0 * s;
        }
#pragma unroll
        for (int a = 0; a < D; ++a) {
            float s = 0.0f;
#pragma unroll
            for (int i = 0; i < D; ++i) s += G[a * D + i] * gx[i];
            T[a][0] = s;
        }
    } else {
        const float lam = c0, mu = c1;
        float Ju[D][D];
#pragma unroll
        for (int s = 0; s < D; ++s)
#pragma unroll
            for (int r = 0; r < D; ++r) {
                float acc = 0.0f;
#pragma unroll
                for (int a = 0; a < D; ++a) acc += G[a * D + s] * g[a][r];
                Ju[s][r] = acc;
            }
        float div = 0.0f;
#pragma unroll
        for (int r = 0; r < D; ++r) div += Ju[r][r];
#pragma unroll
        for (int u = 0; u < D; ++u) {
            float sg[D];
#pragma unroll
            for (int j = 0; j < D; ++j) sg[j] = mu * (Ju[u][j] + Ju[j][u]) + ((u == j) ? lam * div : 0.0f);
#pragma unroll
            for (int a = 0; a < D; ++a) {
                float s = 0.0f;
#pragma unroll
                for (int j = 0; j < D; ++j) s += G[a * D + j] * sg[j];
                T[a][u] = s;
            }
        }
    }
}

// Shared-memory buffers of one CTA (Tc05Vol offsets from a 1024-byte aligned base).
struct Tc05Smem {
    float *Th, *Tl, *Bh, *Bl, *Uh, *Ul, *Sh, *Sl;
};
template <class S>
__device__ __forceinline__ Tc05Smem tc05_smem(unsigned char* raw_base) {
    using L = Tc05Vol<S>;
    const uint32_t raw = smem_u32(raw_base);
    unsigned char* b = raw_base + ((1024u - (raw & 1023u)) & 1023u);
    return {reinterpret_cast<float*>(b), reinterpret_cast<float*>(b + L::OFF_AFL),
            reinterpret_cast<float*>(b + L::OFF_ABH), reinterpret_cast<float*>(b + L::OFF_ABL),
            reinterpret_cast<float*>(b + L::OFF_UH), reinterpret_cast<float*>(b + L::OFF_UL),
            reinterpret_cast<float*>(b + L::OFF_SH), reinterpret_cast<float*>(b + L::OFF_SL)};
}

// Both table copies (hi / lo split) from the FP32 volume table tv (row q D + a, ld ldt), zero past
// Nq and NBF, and S zeroed (rows past Nq stay zero); threads t0, t0 + nt, ...
template <class S>
__device__ void tc05_init(Tc05Smem const& b, const float* __restrict__ tv, int ldt, int Nq, int t0, int nt) {
    using L = Tc05Vol<S>;
    constexpr int D = S::D, NBF = S::NBF, KF = L::KF, KC = L::KC, NQ = L::NQ;
    // forward: core matrices [k/4][a][q/8][8 q][4 k]
    for (int i = t0; i < KC * D * NQ * 4; i += nt) {
        const int kk = i & 3, qq = (i >> 2) & 7, rest = i >> 5;  // rest = (kc * D + a) * 8 + qg
        const int qg = rest & 7, a = (rest >> 3) % D, kc = (rest >> 3) / D;
        const int q = qg * 8 + qq, k = kc * 4 + kk;
        const float v = (q < Nq && k < NBF) ? tv[static_cast<int64_t>(q * D + a) * ldt + k] : 0.0f;
        float h, l;
        split_tf32(v, h, l);
        b.Th[i] = h;
        b.Tl[i] = l;
    }
    // backward: element (k, (a, q)) of the K-major [k][(a, q)] operand
    for (int i = t0; i < KF * L::KB; i += nt) {
        const int k = i % KF, kk = i / KF, a = kk / NQ, q = kk % NQ;
        const float v = (q < Nq && k < NBF) ? tv[static_cast<int64_t>(q * D + a) * ldt + k] : 0.0f;
        float h, l;
        split_tf32(v, h, l);
        const int o = (kk >> 2) * (L::LBO_B / 4) + (k >> 3) * 32 + (k & 7) * 4 + (kk & 3);
        b.Bh[o] = h;
        b.Bl[o] = l;
    }
    for (int i = t0; i < 2 * L::SB / 4; i += nt) b.Sh[i] = 0.0f;  // Sh and Sl are adjacent
}

// U hi / lo of the tile at element e0: one 16-byte K chunk of one column per item, columns fastest;
// items t0, t0 + nt, ...
template <class S, typename TX>
__device__ __forceinline__ void tc05_stage(Tc05Smem const& b, const TX* __restrict__ xr, int64_t e0, int64_t E,
                                           int t0, int nt) {
    using L = Tc05Vol<S>;
    constexpr int NBF = S::NBF, BS = S::BS, TE = L::TE, NCOL = L::NCOL, KC = L::KC;
    for (int i = t0; i < NCOL * KC; i += nt) {
        const int n = i % NCOL, kc = i / NCOL;
        const int r = n / TE, te = n % TE;
        const int64_t e = e0 + te;
        float h[4], l[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k = kc * 4 + j;
            const float v = (e < E && k < NBF) ? static_cast<float>(xr[e * BS + k + NBF * r]) : 0.0f;
            split_tf32(v, h[j], l[j]);
        }
        const int o = core_offset(NCOL, n, kc * 4);
        *reinterpret_cast<float4*>(b.Uh + o) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(b.Ul + o) = make_float4(l[0], l[1], l[2], l[3]);
    }
}

// Forward MMAs (one thread): R_a = D_a U^T into TMEM columns a * NCOL, 3xTF32.
template <class S, int NP = 3>
__device__ __forceinline__ void tc05_issue_fwd(Tc05Smem const& b, uint32_t tmem) {
    using L = Tc05Vol<S>;
    constexpr int NCOL = L::NCOL;
    const uint32_t idf = idesc_tf32(128, NCOL);
    const uint32_t th = smem_u32(b.Th), tl = smem_u32(b.Tl), uh = smem_u32(b.Uh), ul = smem_u32(b.Ul);
    constexpr uint32_t lboU = (NCOL / 8) * 128;
#pragma unroll 1
    for (int a = 0; a < S::D; ++a)
#pragma unroll 1
        for (int s = 0; s < L::KF / 8; ++s) {
            const uint32_t ot = 2u * s * L::KCS + a * 1024u, ou = 2u * s * lboU;
            const uint64_t ah = umma_desc(th + ot, L::KCS, 128), al = umma_desc(tl + ot, L::KCS, 128);
            const uint64_t bh = umma_desc(uh + ou, lboU, 128), bl = umma_desc(ul + ou, lboU, 128);
            const uint32_t d = tmem + static_cast<uint32_t>(a * NCOL);
            umma_tf32(d, ah, bh, idf, s > 0 ? 1u : 0u);
            if constexpr (NP == 3) {
                umma_tf32(d, ah, bl, idf, 1u);
                umma_tf32(d, al, bh, idf, 1u);
            }
        }
}

// Backward MMAs (one thread): Y = D^T S^T into TMEM columns D * NCOL, 3xTF32.
template <class S, int NP = 3>
__device__ __forceinline__ void tc05_issue_bwd(Tc05Smem const& b, uint32_t tmem) {
    using L = Tc05Vol<S>;
    constexpr int NCOL = L::NCOL;
    const uint32_t idb = idesc_tf32(128, NCOL);
    const uint32_t bh0 = smem_u32(b.Bh), bl0 = smem_u32(b.Bl), sh = smem_u32(b.Sh), sl = smem_u32(b.Sl);
    const uint32_t d = tmem + static_cast<uint32_t>(S::D * NCOL);
#pragma unroll 1
    for (int s = 0; s < S::D * L::NQ / 8; ++s) {
        const uint32_t ob = 2u * s * L::LBO_B, os = 2u * s * L::SCS;
        const uint64_t ah = umma_desc(bh0 + ob, L::LBO_B, 128), al = umma_desc(bl0 + ob, L::LBO_B, 128);
        const uint64_t bh = umma_desc(sh + os, L::SCS, 128), bl = umma_desc(sl + os, L::SCS, 128);
        umma_tf32(d, ah, bh, idb, s > 0 ? 1u : 0u);
        if constexpr (NP == 3) {
            umma_tf32(d, ah, bl, idb, 1u);
            umma_tf32(d, al, bh, idb, 1u);
        }
    }
}

// J^-1 and the coefficients of the elements te0 .. te0 + NE - 1 at the thread's point q (coalesced
// over q); zero past Nq and past E.
template <class S, int NE>
__device__ __forceinline__ void tc05_load_geo(DevOp<float> const& op, int q, int64_t e0, int te0,
                                              float (&G)[NE][S::DD], float (&c0)[NE], float (&c1)[NE]) {
    constexpr int DD = S::DD;
    const int Nq = op.Nq;
#pragma unroll
    for (int j = 0; j < NE; ++j) {
        const int64_t e = e0 + te0 + j;
        const bool in = q < Nq && e < op.E;
        const float* vg = op.vG + (in ? e * DD * Nq + q : 0);
#pragma unroll
        for (int c = 0; c < DD; ++c) G[j][c] = in ? vg[c * Nq] : 0.0f;
        if constexpr (S::KIND == kPoisson) {
            c0[j] = in ? op.vCoef[e * Nq + q] : 0.0f;
            c1[j] = 0.0f;
        } else {
            c0[j] = in ? op.vCoef[(e * 2 + 0) * Nq + q] : 0.0f;
            c1[j] = in ? op.vCoef[(e * 2 + 1) * Nq + q] : 0.0f;
        }
    }
}

// The pointwise flux from geometry already in registers (zero geometry gives zero flux).
template <class S, int NE>
__device__ __forceinline__ void tc05_flux(const float (&R)[S::D][S::Q][NE], const float (&G)[NE][S::DD],
                                          const float (&c0)[NE], const float (&c1)[NE],
                                          float (&T)[NE][S::D][S::Q]) {
#pragma unroll
    for (int j = 0; j < NE; ++j) {
        float g[S::D][S::Q];
#pragma unroll
        for (int a = 0; a < S::D; ++a)
#pragma unroll
            for (int r = 0; r < S::Q; ++r) g[a][r] = R[a][r][j];
        vol_point<S>(G[j], c0[j], c1[j], g, T[j]);
    }
}
// ... written to S split hi / lo.
template <class S, int NE>
__device__ __forceinline__ void tc05_write_s(Tc05Smem const& b, int q, int te0, const float (&T)[NE][S::D][S::Q]) {
    using L = Tc05Vol<S>;
    constexpr int D = S::D, Q = S::Q, TE = L::TE, NQ = L::NQ;
#pragma unroll
    for (int j = 0; j < NE; ++j)
#pragma unroll
        for (int a = 0; a < D; ++a) {
            const int kk = a * NQ + q;
            const int ob = (kk >> 2) * (L::SCS / 4) + (kk & 3);
#pragma unroll
            for (int r = 0; r < Q; ++r) {
                const int n = r * TE + te0 + j;
                float h, l;
                split_tf32(T[j][a][r], h, l);
                b.Sh[ob + (n >> 3) * 32 + (n & 7) * 4] = h;
                b.Sl[ob + (n >> 3) * 32 + (n & 7) * 4] = l;
            }
        }
}

// The pointwise flux from geometry already in registers (zero geometry gives zero flux), written to
// S split hi / lo.
template <class S, int NE>
__device__ __forceinline__ void tc05_pointwise_regs(Tc05Smem const& b, int q, int te0, const float (&R)[S::D][S::Q][NE],
                                                    const float (&G)[NE][S::DD], const float (&c0)[NE],
                                                    const float (&c1)[NE]) {
    using L = Tc05Vol<S>;
    constexpr int D = S::D, Q = S::Q, TE = L::TE, NQ = L::NQ;
#pragma unroll
    for (int j = 0; j < NE; ++j) {
        float T[D][Q], g[D][Q];
#pragma unroll
        for (int a = 0; a < D; ++a)
#pragma unroll
            for (int r = 0; r < Q; ++r) g[a][r] = R[a][r][j];
        vol_point<S>(G[j], c0[j], c1[j], g, T);
#pragma unroll
        for (int a = 0; a < D; ++a) {
            const int kk = a * NQ + q;
            const int ob = (kk >> 2) * (L::SCS / 4) + (kk & 3);
#pragma unroll
            for (int r = 0; r < Q; ++r) {
                const int n = r * TE + te0 + j;
                float h, l;
                split_tf32(T[a][r], h, l);
                b.Sh[ob + (n >> 3) * 32 + (n & 7) * 4] = h;
                b.Sl[ob + (n >> 3) * 32 + (n & 7) * 4] = l;
            }
        }
    }
}

// Pointwise flux of the elements te0 .. te0 + NE - 1 at the thread's point q (a lane of 0..63) from
// R[a][r][j], written to S split hi / lo; zero past Nq and past E.
template <class S, int NE>
__device__ __forceinline__ void tc05_pointwise(Tc05Smem const& b, DevOp<float> const& op, int q, int64_t e0, int te0,
                                               const float (&R)[S::D][S::Q][NE]) {
    using L = Tc05Vol<S>;
    constexpr int D = S::D, Q = S::Q, DD = S::DD, TE = L::TE, NQ = L::NQ;
    const int Nq = op.Nq;
#pragma unroll
    for (int j = 0; j < NE; ++j) {
        const int64_t e = e0 + te0 + j;
        float T[D][Q];
        if (q < Nq && e < op.E) {
            float G[DD], g[D][Q];
            const float* vg = op.vG + e * DD * Nq + q;
#pragma unroll
            for (int c = 0; c < DD; ++c) G[c] = vg[c * Nq];
            float c0, c1 = 0.0f;
            if constexpr (S::KIND == kPoisson) {
                c0 = op.vCoef[e * Nq + q];
            } else {
                c0 = op.vCoef[(e * 2 + 0) * Nq + q];
                c1 = op.vCoef[(e * 2 + 1) * Nq + q];
            }
#pragma unroll
            for (int a = 0; a < D; ++a)
#pragma unroll
                for (int r = 0; r < Q; ++r) g[a][r] = R[a][r][j];
            vol_point<S>(G, c0, c1, g, T);
        } else {
#pragma unroll
            for (int a = 0; a < D; ++a)
#pragma unroll
                for (int r = 0; r < Q; ++r) T[a][r] = 0.0f;
        }
#pragma unroll
        for (int a = 0; a < D; ++a) {
            const int kk = a * NQ + q;
            const int ob = (kk >> 2) * (L::SCS / 4) + (kk & 3);
#pragma unroll
            for (int r = 0; r < Q; ++r) {
                const int n = r * TE + te0 + j;
                float h, l;
                split_tf32(T[a][r], h, l);
                b.Sh[ob + (n >> 3) * 32 + (n & 7) * 4] = h;
                b.Sl[ob + (n >> 3) * 32 + (n & 7) * 4] = l;
            }
        }
    }
}

// y of the tile's elements half * 8 .. half * 8 + 7 from the backward accumulator (warp-collective;
// lanes k < NBF store).
template <class S, typename TX>
__device__ __forceinline__ void tc05_store_y4(uint32_t tmem, uint32_t lane_base, int k, int te0, int64_t e0, int64_t E,
                                              TX* __restrict__ yr) {
    using L = Tc05Vol<S>;
    constexpr int Q = S::Q, NBF = S::NBF, BS = S::BS, TE = L::TE, NCOL = L::NCOL;
    float v[Q][4];
#pragma unroll
    for (int r = 0; r < Q; ++r) tmem_ld4(tmem + lane_base + static_cast<uint32_t>(S::D * NCOL + r * TE + te0), v[r]);
    tmem_wait_ld();
    if (k < NBF) {
#pragma unroll
        for (int r = 0; r < Q; ++r)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t e = e0 + te0 + j;
                if (e < E) yr[e * BS + k + NBF * r] = static_cast<TX>(v[r][j]);
            }
    }
}

template <class S, typename TX>
__device__ __forceinline__ void tc05_store_y(uint32_t tmem, uint32_t lane_base, int k, int half, int64_t e0, int64_t E,
                                             TX* __restrict__ yr) {
    using L = Tc05Vol<S>;
    constexpr int Q = S::Q, NBF = S::NBF, BS = S::BS, TE = L::TE, NCOL = L::NCOL;
#pragma unroll
    for (int r = 0; r < Q; ++r) {
        float v[8];
        tmem_ld8(tmem + lane_base + static_cast<uint32_t>(S::D * NCOL + r * TE + half * 8), v);
        tmem_wait_ld();
        if (k < NBF) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int64_t e = e0 + half * 8 + j;
                if (e < E) yr[e * BS + k + NBF * r] = static_cast<TX>(v[j]);
            }
        }
    }
}

// One tile at a time, every phase by the whole CTA (256 threads): stage, forward, pointwise
// (warps owning lanes 0..63), backward, store.  tv: the FP32 volume table, row (q D + a), ld ldt.
// Element tile and right-hand side of work item w (the tile fastest); one right-hand side needs no
// division.
__device__ __forceinline__ int64_t t5_tile(int64_t w, int64_t ntiles, int nrhs) { return nrhs == 1 ? w : w % ntiles; }
__device__ __forceinline__ int64_t t5_rhs(int64_t w, int64_t ntiles, int nrhs) { return nrhs == 1 ? 0 : w / ntiles; }

template <class S, typename TX, int NP = 3>
__global__ void __launch_bounds__(256, 1)
    vol_tc05_kernel(DevOp<float> op, const float* __restrict__ tv, int ldt, const TX* __restrict__ x,
                    TX* __restrict__ y, int64_t ld, int nrhs, int* status) {
    using L = Tc05Vol<S>;
    constexpr int D = S::D, Q = S::Q, TE = L::TE, NCOL = L::NCOL, NT = 256;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long bar;
    __shared__ uint32_t tbase;
    const Tc05Smem b = tc05_smem<S>(smem_raw);
    if (warp == 0) {
        tmem_alloc(&tbase, L::TCOLS);
        tmem_relinquish();
    }
    if (tid == 0) mbar_init(&bar, 1);
    tc05_init<S>(b, tv, ldt, op.Nq, tid, NT);
    fence_async_smem();
    tc05_fence_before();
    __syncthreads();
    tc05_fence_after();
    const uint32_t tmem = tbase;
    const uint32_t lane_base = static_cast<uint32_t>(32 * (warp & 3)) << 16;
    const bool pw = (warp & 3) < 2;  // owns lanes 0..63
    const int half = warp >> 2;
    const int ntiles = static_cast<int>((op.E + TE - 1) / TE);
    const int64_t nwork = static_cast<int64_t>(ntiles) * nrhs;
    unsigned phase = 0;
    bool ok = true;
    for (int64_t work = blockIdx.x; work < nwork && ok; work += gridDim.x) {
        const int64_t e0 = t5_tile(work, ntiles, nrhs) * TE;
        const TX* xr = x + t5_rhs(work, ntiles, nrhs) * ld;
        TX* yr = y + t5_rhs(work, ntiles, nrhs) * ld;
        tc05_stage<S, TX>(b, xr, e0, op.E, tid, NT);
        fence_async_smem();
        tc05_fence_before();
        __syncthreads();
        tc05_fence_after();
        if (tid == 0) {
            tc05_issue_fwd<S, NP>(b, tmem);
            umma_commit(&bar);
        }
        ok = __syncthreads_and(mbar_wait_bounded(&bar, phase) ? 1 : 0) != 0;  // block-uniform
        phase ^= 1u;
        tc05_fence_after();
        if (ok && pw) {
            const int q = 32 * (warp & 3) + lane;
#pragma unroll 1
            for (int g4 = 0; g4 < TE / 8; ++g4) {
                const int te0 = half * (TE / 2) + 4 * g4;
                float R[D][Q][4];
#pragma unroll
                for (int a = 0; a < D; ++a)
#pragma unroll
                    for (int r = 0; r < Q; ++r)
                        tmem_ld4(tmem + lane_base + static_cast<uint32_t>(a * NCOL + r * TE + te0), R[a][r]);
                tmem_wait_ld();
                tc05_pointwise<S, 4>(b, op, q, e0, te0, R);
            }
        }
        fence_async_smem();
        tc05_fence_before();
        __syncthreads();
        tc05_fence_after();
        if (ok && tid == 0) {
            tc05_issue_bwd<S, NP>(b, tmem);
            umma_commit(&bar);
        }
        if (ok) {
            ok = __syncthreads_and(mbar_wait_bounded(&bar, phase) ? 1 : 0) != 0;
            phase ^= 1u;
        }
        tc05_fence_after();
        if (ok && pw) tc05_store_y<S, TX>(tmem, lane_base, 32 * (warp & 3) + lane, half, e0, op.E, yr);
        tc05_fence_before();
        __syncthreads();
    }
    if (!ok && tid == 0 && status) atomicExch(status, 1);
    tc05_fence_after();
    if (warp == 0) tmem_dealloc(tmem, L::TCOLS);
}

// Warp-specialised form (512 threads, 16 warps): in each of the four groups of warps 4g .. 4g + 3,
// the two warps that own TMEM lanes 0..63 run the pointwise flux and the stores of y for elements
// 4g .. 4g + 3 of the tile (lane = point q / basis function k), the other two stage U, except lane 0
// of warp 2, which issues the MMAs.  Five mbarriers, one phase per tile each: U staged (255
// arrivals), forward done (commit), R read (256), S written (256), backward done (commit).  The
// forward MMAs of tile i + 1 are issued as soon as its U is staged and tile i's R has been read, so
// they run under the pointwise phase of tile i; the pointwise threads compute tile i's flux in
// registers while the backward MMAs of tile i - 1 run, and load each tile's geometry before they
// wait for its forward MMAs.  Every wait is bounded; a thread whose wait runs out records the status word and leaves its
// loop, so the threads that wait on it run out in turn and the CTA ends.
template <class S, typename TX, int NP = 3>
__global__ void __launch_bounds__(512, 1)
    vol_tc05p_kernel(DevOp<float> op, const float* __restrict__ tv, int ldt, const TX* __restrict__ x,
                     TX* __restrict__ y, int64_t ld, int nrhs, int* status) {
    using L = Tc05Vol<S>;
    constexpr int D = S::D, Q = S::Q, DD = S::DD, TE = L::TE, NCOL = L::NCOL, NT = 512;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long barU, barF, barR, barS, barB;
    __shared__ uint32_t tbase;
    const Tc05Smem b = tc05_smem<S>(smem_raw);
    if (warp == 0) {
        tmem_alloc(&tbase, L::TCOLS);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&barU, 255);
        mbar_init(&barF, 1);
        mbar_init(&barR, 256);
        mbar_init(&barS, 256);
        mbar_init(&barB, 1);
    }
    tc05_init<S>(b, tv, ldt, op.Nq, tid, NT);
    fence_async_smem();
    tc05_fence_before();
    __syncthreads();
    tc05_fence_after();
    const uint32_t tmem = tbase;
    const int ntiles = static_cast<int>((op.E + TE - 1) / TE);
    const int64_t nwork = static_cast<int64_t>(ntiles) * nrhs;
    const int64_t nmine = nwork > blockIdx.x ? (nwork - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    auto work_of = [&](int64_t i) { return blockIdx.x + i * gridDim.x; };
    const int grp = warp >> 2, sub = warp & 3;
    bool ok = true;
    if (warp == 2 && lane == 0) {  // MMA issue: the forward MMAs of tile i + 1 ahead of the backward of tile i
        if (nmine > 0) {
            ok = mbar_wait_bounded(&barU, 0u);
            if (ok) {
                tc05_fence_after();
                tc05_issue_fwd<S, NP>(b, tmem);
                umma_commit(&barF);
            }
        }
        for (int64_t i = 0; i < nmine && ok; ++i) {
            const unsigned p = static_cast<unsigned>(i & 1);
            if (i + 1 < nmine) {  // U of tile i + 1 staged, R of tile i read
                ok = mbar_wait_bounded(&barU, p ^ 1u) && mbar_wait_bounded(&barR, p);
                if (!ok) break;
                tc05_fence_after();
                tc05_issue_fwd<S, NP>(b, tmem);
                umma_commit(&barF);
            }
            ok = mbar_wait_bounded(&barS, p);
            if (!ok) break;
            tc05_fence_after();
            tc05_issue_bwd<S, NP>(b, tmem);
            umma_commit(&barB);
        }
    } else if (sub >= 2) {  // staging (255 threads): U of tile i once the forward MMAs of tile i - 1 are done
        const int t0 = (grp * 2 + (sub - 2)) * 32 + lane - 1;
        const unsigned mask = warp == 2 ? 0xfffffffeu : 0xffffffffu;
        for (int64_t i = 0; i < nmine && ok; ++i) {
            if (i > 0) ok = __all_sync(mask, mbar_wait_bounded(&barF, static_cast<unsigned>((i - 1) & 1)));
            if (!ok) break;
            const int64_t w = work_of(i);
            tc05_stage<S, TX>(b, x + t5_rhs(w, ntiles, nrhs) * ld, t5_tile(w, ntiles, nrhs) * TE, op.E, t0, 255);
            fence_async_smem();
            mbar_arrive(&barU);
        }
    } else {  // pointwise and stores: lane q / k of 0..63, elements 4 grp .. 4 grp + 3
        const uint32_t lane_base = static_cast<uint32_t>(32 * sub) << 16;
        const int q = 32 * sub + lane, te0 = 4 * grp;
        for (int64_t i = 0; i < nmine && ok; ++i) {
            const unsigned p = static_cast<unsigned>(i & 1);
            const int64_t w = work_of(i);
            const int64_t e0 = t5_tile(w, ntiles, nrhs) * TE;
            float G[4][DD], c0[4], c1[4];
            tc05_load_geo<S, 4>(op, q, e0, te0, G, c0, c1);  // in flight during the wait
            ok = __all_sync(0xffffffffu, mbar_wait_bounded(&barF, p));
            if (!ok) break;
            tc05_fence_after();
            float R[D][Q][4];
#pragma unroll
            for (int a = 0; a < D; ++a)
#pragma unroll
                for (int r = 0; r < Q; ++r)
                    tmem_ld4(tmem + lane_base + static_cast<uint32_t>(a * NCOL + r * TE + te0), R[a][r]);
            tmem_wait_ld();
            tc05_fence_before();
            mbar_arrive(&barR);
            float T[4][D][Q];  // the flux, computed while the previous tile's backward MMAs run
            tc05_flux<S, 4>(R, G, c0, c1, T);
            if (i > 0) {  // the previous tile's y (its backward MMAs also released S)
                ok = __all_sync(0xffffffffu, mbar_wait_bounded(&barB, p ^ 1u));
                if (!ok) break;
                tc05_fence_after();
                const int64_t wp = work_of(i - 1);
                tc05_store_y4<S, TX>(tmem, lane_base, q, te0, t5_tile(wp, ntiles, nrhs) * TE, op.E,
                                     y + t5_rhs(wp, ntiles, nrhs) * ld);
                tc05_fence_before();
            }
            tc05_write_s<S, 4>(b, q, te0, T);
            fence_async_smem();
            mbar_arrive(&barS);
        }
        if (ok && nmine > 0) {
            ok = __all_sync(0xffffffffu, mbar_wait_bounded(&barB, static_cast<unsigned>((nmine - 1) & 1)));
            if (ok) {
                tc05_fence_after();
                const int64_t wp = work_of(nmine - 1);
                tc05_store_y4<S, TX>(tmem, lane_base, q, te0, t5_tile(wp, ntiles, nrhs) * TE, op.E,
                                     y + t5_rhs(wp, ntiles, nrhs) * ld);
            }
        }
    }
    if (!ok && status) atomicExch(status, 1);
    tc05_fence_before();
    __syncthreads();
    tc05_fence_after();
    if (warp == 0) tmem_dealloc(tmem, L::TCOLS);
}

}  // namespace tdg
