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
//     (MN-major, one 16-byte store per 4 elements) split hi / lo;
//  4. backward: Y[k][n] = sum_(a, q) D_a[q][k] S[n][(a, q)] into TMEM (M = 128 lanes = basis k,
//     K = D * 64; the table read MN-major through a second descriptor over the same copy);
//  5. y: lanes k < NBF store y[e BS + k + NBF r] (32 consecutive k per warp store).
//
// The table D_a[q][k] lives once per CTA in shared memory as core matrices [k/4][a][q/8][8 q][4 k]
// (hi and lo copies), read K-major by the forward MMA (rows q: SBO 128 bytes, K chunks: LBO D KB)
// and MN-major by the backward MMA (rows k in groups of 4: SBO D KB, K groups (a, q/8): LBO 128
// bytes).  Rows of an M = 128 operand past the stored ones read other shared memory; they only
// produce accumulator rows that are never read, and the buffer is sized so that every such read
// stays inside it.
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
    static constexpr int KCS = D * NQ * 16;          // bytes between K chunks of the table
    static constexpr int TAB = KC * KCS;             // bytes of one table copy
    static constexpr int UB = NCOL * KF * 4;         // bytes of one U copy
    static constexpr int SB = NCOL * KB * 4;         // bytes of one S copy
    static constexpr int OFF_TL = TAB, OFF_UH = 2 * TAB, OFF_UL = OFF_UH + UB, OFF_SH = OFF_UL + UB,
                         OFF_SL = OFF_SH + SB, END = OFF_SL + SB;
    // last byte the backward MMA's 32 m-groups can reach from the lo table, plus the forward's
    // 16 q-groups past the last block
    static constexpr int REACH = OFF_TL + 32 * KCS + 2048;
    static constexpr int BYTES = (END > REACH ? END : REACH) + 1024;  // + alignment
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

// tv: the FP32 volume table of the tensor kernels, row (q D + a), ld = ldt, columns k < NBF.
template <class S, typename TX>
__global__ void __launch_bounds__(256, 1)
    vol_tc05_kernel(DevOp<float> op, const float* __restrict__ tv, int ldt, const TX* __restrict__ x,
                    TX* __restrict__ y, int64_t ld, int nrhs, int* status) {
    using L = Tc05Vol<S>;
    constexpr int D = S::D, Q = S::Q, NBF = S::NBF, BS = S::BS, DD = S::DD;
    constexpr int TE = L::TE, NCOL = L::NCOL, KF = L::KF, KC = L::KC, NQ = L::NQ, NT = L::NT;
    const int Nq = op.Nq;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long bar;
    __shared__ uint32_t tbase;
    const uint32_t raw = smem_u32(smem_raw);
    unsigned char* base = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
    float* Th = reinterpret_cast<float*>(base);
    float* Tl = reinterpret_cast<float*>(base + L::OFF_TL);
    float* Uh = reinterpret_cast<float*>(base + L::OFF_UH);
    float* Ul = reinterpret_cast<float*>(base + L::OFF_UL);
    float* Sh = reinterpret_cast<float*>(base + L::OFF_SH);
    float* Sl = reinterpret_cast<float*>(base + L::OFF_SL);
    if (warp == 0) {
        tmem_alloc(&tbase, L::TCOLS);
        tmem_relinquish();
    }
    if (tid == 0) mbar_init(&bar, 1);
    // the table D_a[q][k] as core matrices [k/4][a][q/8][8][4], zero past Nq and NBF
    for (int i = tid; i < KC * D * NQ * 4; i += NT) {
        const int kk = i & 3, qq = (i >> 2) & 7, rest = i >> 5;  // rest = (kc * D + a) * 8 + qg
        const int qg = rest & 7, a = (rest >> 3) % D, kc = (rest >> 3) / D;
        const int q = qg * 8 + qq, k = kc * 4 + kk;
        const float v = (q < Nq && k < NBF) ? tv[static_cast<int64_t>(q * D + a) * ldt + k] : 0.0f;
        float h, l;
        split_tf32(v, h, l);
        Th[i] = h;
        Tl[i] = l;
    }
    // S starts (and stays, past Nq) zero
    for (int i = tid; i < 2 * NCOL * L::KB; i += NT) Sh[i] = 0.0f;  // Sh and Sl are adjacent
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
        const int tile = static_cast<int>(work % ntiles);
        const TX* xr = x + (work / ntiles) * ld;
        TX* yr = y + (work / ntiles) * ld;
        const int64_t e0 = static_cast<int64_t>(tile) * TE;
        // 1. U hi / lo: one 16-byte K chunk of one column per item, columns fastest
        for (int i = tid; i < NCOL * KC; i += NT) {
            const int n = i % NCOL, kc = i / NCOL;
            const int r = n / TE, te = n % TE;
            const int64_t e = e0 + te;
            float v[4], h[4], l[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int k = kc * 4 + j;
                v[j] = (e < op.E && k < NBF) ? static_cast<float>(xr[e * BS + k + NBF * r]) : 0.0f;
                split_tf32(v[j], h[j], l[j]);
            }
            const int o = core_offset(NCOL, n, kc * 4);
            *reinterpret_cast<float4*>(Uh + o) = make_float4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<float4*>(Ul + o) = make_float4(l[0], l[1], l[2], l[3]);
        }
        fence_async_smem();
        tc05_fence_before();
        __syncthreads();
        tc05_fence_after();
        // 2. forward MMAs
        if (tid == 0) {
            const uint32_t idf = idesc_tf32(128, NCOL);
            const uint32_t th = smem_u32(Th), tl = smem_u32(Tl), uh = smem_u32(Uh), ul = smem_u32(Ul);
            constexpr uint32_t lboU = (NCOL / 8) * 128;
#pragma unroll 1
            for (int a = 0; a < D; ++a)
#pragma unroll 1
                for (int s = 0; s < KF / 8; ++s) {
                    const uint32_t ot = 2u * s * L::KCS + a * 1024u, ou = 2u * s * lboU;
                    const uint64_t ah = umma_desc(th + ot, L::KCS, 128), al = umma_desc(tl + ot, L::KCS, 128);
                    const uint64_t bh = umma_desc(uh + ou, lboU, 128), bl = umma_desc(ul + ou, lboU, 128);
                    const uint32_t d = tmem + static_cast<uint32_t>(a * NCOL);
                    umma_tf32(d, ah, bh, idf, s > 0 ? 1u : 0u);
                    umma_tf32(d, ah, bl, idf, 1u);
                    umma_tf32(d, al, bh, idf, 1u);
                }
            umma_commit(&bar);
        }
        ok = __syncthreads_and(mbar_wait_bounded(&bar, phase) ? 1 : 0) != 0;  // block-uniform
        phase ^= 1u;
        tc05_fence_after();
        // 3. pointwise (warps owning lanes 0..63); lanes past Nq and elements past E give zero S
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
                float T[D][Q][4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int64_t e = e0 + te0 + j;
                    float Tj[D][Q];
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
                        vol_point<S>(G, c0, c1, g, Tj);
                    } else {
#pragma unroll
                        for (int a = 0; a < D; ++a)
#pragma unroll
                            for (int r = 0; r < Q; ++r) Tj[a][r] = 0.0f;
                    }
#pragma unroll
                    for (int a = 0; a < D; ++a)
#pragma unroll
                        for (int r = 0; r < Q; ++r) T[a][r][j] = Tj[a][r];
                }
#pragma unroll
                for (int a = 0; a < D; ++a)
#pragma unroll
                    for (int r = 0; r < Q; ++r) {
                        const int o = core_offset_mn(NCOL, r * TE + te0, a * NQ + q);
                        float h[4], l[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j) split_tf32(T[a][r][j], h[j], l[j]);
                        *reinterpret_cast<float4*>(Sh + o) = make_float4(h[0], h[1], h[2], h[3]);
                        *reinterpret_cast<float4*>(Sl + o) = make_float4(l[0], l[1], l[2], l[3]);
                    }
            }
        }
        fence_async_smem();
        tc05_fence_before();
        __syncthreads();
        tc05_fence_after();
        // 4. backward MMAs: the table read MN-major (rows k), S MN-major
        if (ok && tid == 0) {
            const uint32_t idb = idesc_tf32(128, NCOL, true, true);
            const uint32_t th = smem_u32(Th), tl = smem_u32(Tl), sh = smem_u32(Sh), sl = smem_u32(Sl);
            constexpr uint32_t lboS = (NCOL / 4) * 128;
            const uint32_t d = tmem + static_cast<uint32_t>(D * NCOL);
#pragma unroll 1
            for (int s = 0; s < D * NQ / 8; ++s) {
                const uint64_t ah = umma_desc(th + 128u * s, 128, L::KCS), al = umma_desc(tl + 128u * s, 128, L::KCS);
                const uint64_t bh = umma_desc(sh + lboS * s, lboS, 128), bl = umma_desc(sl + lboS * s, lboS, 128);
                umma_tf32(d, ah, bh, idb, s > 0 ? 1u : 0u);
                umma_tf32(d, ah, bl, idb, 1u);
                umma_tf32(d, al, bh, idb, 1u);
            }
            umma_commit(&bar);
        }
        if (ok) {
            ok = __syncthreads_and(mbar_wait_bounded(&bar, phase) ? 1 : 0) != 0;
            phase ^= 1u;
        }
        tc05_fence_after();
        // 5. y = Y (lanes k < NBF; each half of the warps stores half of the tile's elements)
        if (ok && pw) {
            const int k = 32 * (warp & 3) + lane;
#pragma unroll
            for (int r = 0; r < Q; ++r) {
                float v[8];
                tmem_ld8(tmem + lane_base + static_cast<uint32_t>(D * NCOL + r * TE + half * 8), v);
                tmem_wait_ld();
                if (k < NBF) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int64_t e = e0 + half * 8 + j;
                        if (e < op.E) yr[e * BS + k + NBF * r] = static_cast<TX>(v[j]);
                    }
                }
            }
        }
        tc05_fence_before();
        __syncthreads();
    }
    if (!ok && tid == 0 && status) atomicExch(status, 1);
    tc05_fence_after();
    if (warp == 0) tmem_dealloc(tmem, L::TCOLS);
}

}  // namespace tdg
