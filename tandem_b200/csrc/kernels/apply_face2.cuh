// Face-centric FP64 apply, software-pipelined: the operator of apply_face.cuh (volume kernel +
// one pass over the facets, tandem's apply_volume / flux / apply_facet einsums,
// app/kernels/elasticity.py:201-234, poisson.py:123-140; the facet loop of Poisson.cpp:586-631 and
// Elasticity.cpp:734-801 with every facet evaluated once for both sides) with the memory traffic of
// a tile taken off the critical path:
//
//  * the coefficient blocks of the next tile are copied into shared memory with cp.async while the
//    current tile computes (double buffer), element-major as x holds them -- each element's Q
//    component runs of Nbf values land at a component stride KS and an element stride LDU chosen
//    so that the m8n8k4 B-fragment loads of every half warp hit 16 distinct 8-byte banks;
//  * the per-point geometry and coefficients are read from copies laid out per tile, point-major
//    with the tile's elements (or facets) fastest, so the pointwise phase's loads are coalesced;
//  * the facet flux evaluates the averaged stress once for both sides (the side-1 view of tandem's
//    flux, Elasticity.cpp:734-747, shares it: the side-1 value row is the negated side-0 row and the
//    gradient rows differ only in the side's J^-1 and Lame parameters).
//
// The tables (basis derivatives / values at the points) and the GEMM tiling are those of
// apply_mma.cuh.  Results agree with the other FP64 kernels to rounding (atomics into y).
#pragma once

#include "apply_face.cuh"
#include "async.cuh"

namespace tdg {

// ---- staged coefficient blocks --------------------------------------------------------------------

// True when the B-fragment addresses (k = t, n = nt * 8 + g; address (n / Q) * ldu + (n % Q) * ks
// + k) of both half warps are distinct modulo 16 doubles, for every n-tile.
__host__ __device__ constexpr bool staged_conflict_free(int Q, int ks, int ldu, int ntn) {
    for (int nt = 0; nt < ntn; ++nt)
        for (int half = 0; half < 2; ++half) {
            bool used[16] = {};
            for (int g = 4 * half; g < 4 * half + 4; ++g)
                for (int t = 0; t < 4; ++t) {
                    const int n = nt * 8 + g;
                    const int a = ((n / Q) * ldu + (n % Q) * ks + t) % 16;
                    if (used[a]) return false;
                    used[a] = true;
                }
        }
    return true;
}

// Element stride of the staged blocks: the smallest >= Q * ks (at most 16 more) that is conflict
// free, else Q * ks + 4.
__host__ __device__ constexpr int staged_ldu(int Q, int ks, int ntn) {
    for (int l = Q * ks; l < Q * ks + 16; ++l)
        if (staged_conflict_free(Q, ks, l, ntn)) return l;
    return Q * ks + 4;
}

// Component stride: the padded Nbf, or 4, 8 or 12 more where no element stride is conflict free
// with it (2D p4 elasticity: a stride of 16 puts both components' k on the same banks).
__host__ __device__ constexpr int staged_ks(int Q, int kp, int ntn) {
    for (int ks = kp; ks < kp + 16; ks += 4)
        if (staged_conflict_free(Q, ks, staged_ldu(Q, ks, ntn), ntn)) return ks;
    return kp;
}

template <class S>
struct Staged {
    using L = MmaTile<S>;
    static constexpr int KS = staged_ks(S::Q, L::KP, L::NTN);       // component stride
    static constexpr int LDU = staged_ldu(S::Q, KS, L::NTN);       // element stride
    static constexpr int UE = (L::NP + S::Q - 1) / S::Q;           // elements per staged tile
    static constexpr int USZ = UE * LDU;                           // doubles per staged tile
};

// C[M x NP] = A[M x K] U for rows [0, mrows), U staged element-major (Staged<S>): as
// cta_gemm_store with the B fragments read from the staged layout.  Two GEMMs of the same shape
// at once when A1 != nullptr (C1 = A1 U1).
// A load of a table entry: read-only global path (L1) for tables left in global memory, else shared.
template <bool AG>
__device__ __forceinline__ double table_ld(const double* p) {
    if constexpr (AG)
        return __ldg(p);
    else
        return *p;
}

template <class S, int CH = 8, bool AG = false>
__device__ __forceinline__ void cta_gemm_store_staged(const double* A0, const double* U0, double* C0,
                                                      const double* A1, const double* U1, double* C1, int mrows,
                                                      int ksteps, int warp, int lane) {
    using L = MmaTile<S>;
    using SU = Staged<S>;
    constexpr int Q = S::Q;
    const int g = lane >> 2, t = lane & 3;
    const int per = (mrows / 8) * L::NTN;
    const int ntiles = A1 ? 2 * per : per;
    // a warp advances up to CH of its output tiles together (independent accumulators)
    for (int t0 = warp; t0 < ntiles; t0 += CH * L::GW) {
        double acc[CH][2];
        const double* ap[CH];
        const double* bp[CH];
        int cnt = 0;
#pragma unroll
        for (int j = 0; j < CH; ++j) {
            acc[j][0] = acc[j][1] = 0.0;
            const int tile = t0 + j * L::GW;
            const int tt = tile < ntiles ? tile : t0;
            const int which = tt / per, loc = tt % per;
            const int mt = loc / L::NTN, nt = loc % L::NTN;
            const int n = nt * 8 + g;
            ap[j] = (which ? A1 : A0) + (mt * 8 + g) * L::LDT + t;
            bp[j] = (which ? U1 : U0) + (n / Q) * SU::LDU + (n % Q) * SU::KS + t;
            cnt += tile < ntiles;
        }
        for (int ks = 0; ks < ksteps; ++ks) {
#pragma unroll
            for (int j = 0; j < CH; ++j)
                if (j < cnt) dmma(acc[j], table_ld<AG>(ap[j] + ks * 4), bp[j][ks * 4]);
        }
#pragma unroll
        for (int j = 0; j < CH; ++j) {
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

// The same product with register blocking over whole rows of output tiles: a warp's work item is
// one m-tile and all NTN n-tiles of it, so each k step loads one A fragment and NTN B fragments
// for NTN mma (1 + 1/NTN shared-memory loads per mma instead of 2).
template <class S, bool AG = false>
__device__ __forceinline__ void cta_gemm_store_rows(const double* A0, const double* U0, double* C0, const double* A1,
                                                    const double* U1, double* C1, int mrows, int ksteps, int warp,
                                                    int lane) {
    using L = MmaTile<S>;
    using SU = Staged<S>;
    constexpr int Q = S::Q, NTN = L::NTN;
    const int g = lane >> 2, t = lane & 3;
    const int per = mrows / 8;
    const int nitems = A1 ? 2 * per : per;
    for (int it = warp; it < nitems; it += L::GW) {
        const int which = it / per, mt = it % per;
        const double* ap = (which ? A1 : A0) + (mt * 8 + g) * L::LDT + t;
        const double* ub = which ? U1 : U0;
        const double* bp[NTN];
#pragma unroll
        for (int j = 0; j < NTN; ++j) {
            const int n = j * 8 + g;
            bp[j] = ub + (n / Q) * SU::LDU + (n % Q) * SU::KS + t;
        }
        double acc[NTN][2];
#pragma unroll
        for (int j = 0; j < NTN; ++j) acc[j][0] = acc[j][1] = 0.0;
        for (int ks = 0; ks < ksteps; ++ks) {
            const double a = table_ld<AG>(ap + ks * 4);
#pragma unroll
            for (int j = 0; j < NTN; ++j) dmma(acc[j], a, bp[j][ks * 4]);
        }
        double* c = (which ? C1 : C0) + (mt * 8 + g) * L::LDN + 2 * t;  // 16-byte aligned (LDN, 2t even)
#pragma unroll
        for (int j = 0; j < NTN; ++j) *reinterpret_cast<double2*>(c + j * 8) = make_double2(acc[j][0], acc[j][1]);
    }
}

// D (16 x 8) += A (16 x 4) B (4 x 8) in FP64: a0 / a1 = A[g][t] / A[g + 8][t], b = B[t][g],
// d0, d1 = D[g][2t, 2t + 1], d2, d3 = D[g + 8][2t, 2t + 1] (g = lane / 4, t = lane % 4).
__device__ __forceinline__ void dmma16(double (&c)[4], double a0, double a1, double b) {
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b));
}

// cta_gemm_store_rows on 16-row m-tiles (m16n8k4: two A fragments and NTN B fragments per k step
// for NTN mma of twice the work); mrows a multiple of 16.
template <class S, bool AG = false>
__device__ __forceinline__ void cta_gemm_store_rows16(const double* A0, const double* U0, double* C0, const double* A1,
                                                      const double* U1, double* C1, int mrows, int ksteps, int warp,
                                                      int lane) {
    using L = MmaTile<S>;
    using SU = Staged<S>;
    constexpr int Q = S::Q, NTN = L::NTN;
    const int g = lane >> 2, t = lane & 3;
    const int per = mrows / 16;
    const int nitems = A1 ? 2 * per : per;
    for (int it = warp; it < nitems; it += L::GW) {
        const int which = it / per, mt = it % per;
        const double* ap = (which ? A1 : A0) + (mt * 16 + g) * L::LDT + t;
        const double* ub = which ? U1 : U0;
        const double* bp[NTN];
#pragma unroll
        for (int j = 0; j < NTN; ++j) {
            const int n = j * 8 + g;
            bp[j] = ub + (n / Q) * SU::LDU + (n % Q) * SU::KS + t;
        }
        double acc[NTN][4];
#pragma unroll
        for (int j = 0; j < NTN; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
        for (int ks = 0; ks < ksteps; ++ks) {
            const double a0 = table_ld<AG>(ap + ks * 4), a1 = table_ld<AG>(ap + 8 * L::LDT + ks * 4);
#pragma unroll
            for (int j = 0; j < NTN; ++j) dmma16(acc[j], a0, a1, bp[j][ks * 4]);
        }
        double* c = (which ? C1 : C0) + (mt * 16 + g) * L::LDN + 2 * t;
#pragma unroll
        for (int j = 0; j < NTN; ++j) {
            c[j * 8] = acc[j][0];
            c[j * 8 + 1] = acc[j][1];
            c[8 * L::LDN + j * 8] = acc[j][2];
            c[8 * L::LDN + j * 8 + 1] = acc[j][3];
        }
    }
}

// Y += A^T B as cta_gemm_acc_t (apply_mma.cuh), the table A read through table_ld<AG>.
template <class L, bool AG>
__device__ __forceinline__ void cta_gemm_acc_t_tab(const double* A, const double* B, double (&y)[L::YPW][2][2],
                                                   int krows, int warp, int lane) {
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
                if (on[j]) dmma(y[j][h], table_ld<AG>(ac[j] + (ks + h) * 4 * L::LDT), bc[j][(ks + h) * 4 * L::LDN]);
    }
    if (ks < ks_n) {
#pragma unroll
        for (int j = 0; j < L::YPW; ++j)
            if (on[j]) dmma(y[j][0], table_ld<AG>(ac[j] + ks * 4 * L::LDT), bc[j][ks * 4 * L::LDN]);
    }
}

// The facet kernel's face tables: read from global memory through the L1 (true) or copied into
// shared memory per (l0, l1) pair (false).
constexpr bool kFaceTablesGlobal = false;
// Bulk-copy prefetch of each facet tile's geometry into shared memory: 0 never, 1 where it still
// fits two CTAs per SM, 2 always (then one CTA per SM where it does not).
constexpr int kFacetGeometryPrefetch = 1;

// Output tiles a warp advances together in the trace GEMMs (independent accumulators).  Measured on
// the 32^3 p4 elasticity apply (B200, 2 CTAs per SM, 16 warps per SM): volume 1 / facets 2 ran
// 3.10 ms, 4 / 4 3.25 ms, 8 / 8 3.75 ms -- with 16 warps per SM the other warps hide the mma
// latency, and more chains per warp only add live registers and shared-memory traffic in flight.
constexpr int kVolChains = 1;
constexpr int kFaceChains = 2;
// Forward products register-blocked over whole rows of output tiles (cta_gemm_store_rows): measured
// on the same 32^3 apply 3.044 -> 2.844 ms (2 CTAs per SM), the same results bit for bit.
constexpr bool kGemmRows = true;
// The row-blocked forward products on 16-row m-tiles (m16n8k4) where the rows allow it.
constexpr bool kGemmRows16 = false;

// cp.async issue of the coefficient blocks: one (side, element) block per warp with the lanes along
// the block (true), or one flat index per thread over all blocks (false).  Measured on the 32^3
// apply: 2.860 -> 2.789 ms (less index arithmetic per copy).
constexpr bool kStageByWarp = true;

// Issues the cp.async copies of the coefficient blocks of up to UE elements (el[te] < 0: skipped)
// from xr into the staged buffer U.
template <class S, int NT>
__device__ __forceinline__ void stage_blocks(const double* __restrict__ xr, const int* el, double* U, int tid) {
    using SU = Staged<S>;
    constexpr int per_el = S::Q * S::NBF;
    if constexpr (kStageByWarp) {  // one element block per warp, lanes along the block
        const int warp = tid >> 5, lane = tid & 31;
        for (int te = warp; te < SU::UE; te += NT / 32) {
            const int e = el[te];
            if (e < 0) continue;
            double* dst = U + te * SU::LDU;
            const double* src = xr + static_cast<int64_t>(e) * S::BS;
            for (int w = lane; w < per_el; w += 32) cp_async8(dst + (w / S::NBF) * SU::KS + (w % S::NBF), src + w);
        }
        return;
    }
    for (int i = tid; i < SU::UE * per_el; i += NT) {
        const int te = i / per_el, w = i % per_el;
        const int r = w / S::NBF, k = w % S::NBF;
        const int e = el[te];
        if (e >= 0) cp_async8(U + te * SU::LDU + r * SU::KS + k, xr + static_cast<int64_t>(e) * S::BS + w);
    }
}

// (tile, right-hand side) of work item `work` in the per-RHS sweep order (the tile fastest).  The
// kernels call this several times per tile and are issue-bound, so one right-hand side needs no
// division (the kernels' ONE instances, launched for nrhs = 1, fold it away) and 32-bit division
// serves every item count below 2^32.
__device__ __forceinline__ void sweep_tile_rhs(int64_t work, int64_t ntiles, int nrhs, int64_t& tile, int64_t& rhs) {
    if (nrhs == 1) {
        tile = work;
        rhs = 0;
    } else if (static_cast<uint64_t>(ntiles) * static_cast<uint64_t>(nrhs) <= 0xffffffffull) {
        const uint32_t w = static_cast<uint32_t>(work), n = static_cast<uint32_t>(ntiles);
        const uint32_t r = w / n;
        rhs = r;
        tile = w - r * n;
    } else {
        rhs = work / ntiles;
        tile = work - rhs * ntiles;
    }
}

// ---- tile-ordered geometry ------------------------------------------------------------------------

// Volume data per element tile, [tile][field][q][te] with fields J^-1 (DD) then the coefficients
// (Poisson |J| W K; elasticity lam W |J|, mu W |J|): the tile's elements are fastest.
// Facet data per facet tile, [tile][field][q][te] with fields n (D), n_unit (D), then Poisson
// K G0, K G1 (DD each) or elasticity G0, G1 (DD each), lam0, mu0, lam1, mu1; penalty [tile][te].
struct TileGeo {
    const double* vol = nullptr;
    const double* fct = nullptr;
    const double* pen = nullptr;
    int* status = nullptr;  // device word: non-zero once a bounded wait of the facet kernel ran out
};

template <class S>
__host__ __device__ constexpr int vol_fields() {
    return S::DD + (S::KIND == kPoisson ? 1 : 2);
}
template <class S>
__host__ __device__ constexpr int fct_fields() {
    return 2 * S::D + 2 * S::DD + (S::KIND == kPoisson ? 0 : 4);
}

// Points of a tile's geometry rows (volume and facet kernels): with 8 elements / facets per tile
// (3D elasticity) the points are stored in quads with the middle two swapped (row r holds point
// face2_point(r)), so that the pointwise phases' half warps (rows 4c, 4c + 1 or 4c + 2, 4c + 3:
// points two apart) read and write the product rows on disjoint banks while still reading the
// geometry rows contiguously; rows per field: the point count rounded up to the quad.  Other tiles
// keep the points in order.
template <class S>
__host__ __device__ constexpr bool face2_point_swizzle() {
    return MmaTile<S>::TE == 8;
}
template <class S>
__host__ __device__ inline int face2_geo_rows(int nq) {
    return face2_point_swizzle<S>() ? (nq + 3) / 4 * 4 : nq;
}
__host__ __device__ inline int face2_point(int r) { return (r & ~3) | ((r & 1) << 1) | ((r >> 1) & 1); }

// ---- volume kernel ----------------------------------------------------------------------------------

// qc: volume points per pass (all Nq where the buffer fits two CTAs per SM, else MmaTile::QC, or the
// autotuner's pick); fewer passes mean fewer barriers per tile and more pointwise items per pass.
// Every pass but the last starts its table rows on an 8-row mma tile (qc * D rows) and its points on
// a quad of swizzled points, so qc is a multiple of face2_pass_step(D) (dispatch.hpp).
template <class S>
struct Vol2Layout {
    int MV, qc, off_U, off_R, total;
};
template <class S>
__host__ __device__ inline Vol2Layout<S> vol2_layout(int Nq, int qc) {
    using L = MmaTile<S>;
    Vol2Layout<S> l;
    l.MV = round8(S::D * Nq);
    l.qc = qc;
    l.off_U = l.MV * L::LDT;
    l.off_R = l.off_U + 2 * Staged<S>::USZ;
    l.total = l.off_R + round8(qc * S::D) * L::LDN;
    return l;
}
template <class S>
__host__ inline Vol2Layout<S> vol2_layout_auto(int Nq) {
    const Vol2Layout<S> full = vol2_layout<S>(Nq, Nq);
    return full.total * sizeof(double) <= 112 * 1024 ? full : vol2_layout<S>(Nq, MmaTile<S>::QC);
}

template <class S, bool ONE = false>
__global__ void __launch_bounds__(MmaTile<S>::NT, 2)
    vol2_kernel(DevOp<double> op, TileGeo tg, const double* __restrict__ tv, const double* __restrict__ x,
                double* __restrict__ y, int64_t ld, int nrhs, int qc) {
    using L = MmaTile<S>;
    using SU = Staged<S>;
    constexpr int D = S::D, NBF = S::NBF, Q = S::Q, BS = S::BS, DD = S::DD;
    constexpr int TE = L::TE, NT = L::NT, LDN = L::LDN, LDT = L::LDT;
    constexpr int NFLD = vol_fields<S>();
    const int Nq = op.Nq;
    const int Nqg = face2_geo_rows<S>(Nq);  // geometry rows per field
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Vol2Layout<S> lay = vol2_layout<S>(Nq, qc);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sm = reinterpret_cast<double*>(smem_raw);
    double* TV = sm;
    double* Ub = sm + lay.off_U;
    double* R0 = sm + lay.off_R;
    __shared__ int s_el[2][SU::UE];
    for (int i = tid; i < lay.MV * LDT; i += NT) sm[i] = tv[i];
    for (int i = tid; i < 2 * SU::USZ; i += NT) Ub[i] = 0.0;  // padding stays zero, stale columns finite

    const int64_t ntiles = (op.E + TE - 1) / TE;
    const int64_t nwork = ntiles * nrhs;
    auto stage = [&](int64_t work, int buf) {
        int64_t tile, rhs;
        sweep_tile_rhs(work, ntiles, ONE ? 1 : nrhs, tile, rhs);
        const double* xr = x + rhs * ld;
        if (tid < SU::UE) {
            const int64_t e = tile * TE + tid;
            s_el[buf][tid] = (tid < TE && e < op.E) ? static_cast<int>(e) : -1;
        }
        __syncthreads();
        stage_blocks<S, NT>(xr, s_el[buf], Ub + buf * SU::USZ, tid);
        cp_async_commit();
    };
    __syncthreads();
    int buf = 0;
    if (static_cast<int64_t>(blockIdx.x) < nwork) stage(blockIdx.x, 0);
    for (int64_t work = blockIdx.x; work < nwork; work += gridDim.x, buf ^= 1) {
        int64_t tile, rhs;
        sweep_tile_rhs(work, ntiles, ONE ? 1 : nrhs, tile, rhs);
        double* yr = y + rhs * ld;
        const int64_t next = work + gridDim.x;
        __syncthreads();  // the previous tile is done with the other buffer
        if (next < nwork) {
            stage(next, buf ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double* U = Ub + buf * SU::USZ;
        const int* el = s_el[buf];
        const double* geo = tg.vol + tile * static_cast<int64_t>(NFLD) * Nqg * TE;
        double yacc[L::YPW][2][2];
#pragma unroll
        for (int j = 0; j < L::YPW; ++j) yacc[j][0][0] = yacc[j][0][1] = yacc[j][1][0] = yacc[j][1][1] = 0.0;
        for (int q0 = 0; q0 < Nq; q0 += qc) {
            const int nqc = (Nq - q0 < qc) ? (Nq - q0) : qc;
            const int rows = round8(nqc * D);
            if (kGemmRows16 && rows % 16 == 0)
                cta_gemm_store_rows16<S>(TV + q0 * D * LDT, U, R0, nullptr, nullptr, nullptr, rows, L::KP / 4, warp,
                                         lane);
            else if constexpr (kGemmRows)
                cta_gemm_store_rows<S>(TV + q0 * D * LDT, U, R0, nullptr, nullptr, nullptr, rows, L::KP / 4, warp, lane);
            else
                cta_gemm_store_staged<S, kVolChains>(TV + q0 * D * LDT, U, R0, nullptr, nullptr, nullptr, rows,
                                                     L::KP / 4, warp, lane);
            __syncthreads();
            // chunk starts are multiples of 4, so a chunk's rows hold exactly its points
            const int nrow = face2_point_swizzle<S>() ? (nqc + 3) / 4 * 4 : nqc;
            for (int it = tid; it < TE * nrow; it += NT) {
                const int te = it % TE, row = q0 + it / TE;
                const int q = face2_point_swizzle<S>() ? face2_point(row) : row, qq = q - q0;
                if (q >= Nq || el[te] < 0) continue;
                const double* gp = geo + static_cast<int64_t>(row) * TE + te;  // field f at gp[f * Nqg * TE]
                double G[DD];
#pragma unroll
                for (int c = 0; c < DD; ++c) G[c] = gp[static_cast<int64_t>(c) * Nqg * TE];
                double* rr = R0 + (qq * D) * LDN + te * Q;
                if constexpr (S::KIND == kPoisson) {
                    const double jwk = gp[static_cast<int64_t>(DD) * Nqg * TE];
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
                    const double lam = gp[static_cast<int64_t>(DD) * Nqg * TE];
                    const double mu = gp[static_cast<int64_t>(DD + 1) * Nqg * TE];
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
                        const int e = el[te];
                        if (e >= 0) yr[static_cast<int64_t>(e) * BS + k + NBF * r] = yacc[j][0][h] + yacc[j][1][h];
                    }
                }
            }
        }
    }
    cp_async_wait<0>();
}

// ---- facet kernel -----------------------------------------------------------------------------------

template <class S>
struct Face2Layout {
    int MF, off_TB, off_U, off_R0, off_R1, off_G, total;
};
// gpre: room for the current facet tile's geometry, prefetched by the bulk-copy engine.
template <class S>
__host__ __device__ inline Face2Layout<S> face2_layout(int nq, int gpre = 0) {
    using L = MmaTile<S>;
    Face2Layout<S> l;
    l.MF = round8((S::D + 1) * nq);
    l.off_TB = kFaceTablesGlobal ? 0 : l.MF * L::LDT;
    l.off_U = kFaceTablesGlobal ? 0 : l.off_TB + l.MF * L::LDT;
    l.off_R0 = l.off_U + 4 * Staged<S>::USZ;  // [buffer][side]
    l.off_R1 = l.off_R0 + l.MF * L::LDN;
    l.off_G = l.off_R1 + l.MF * L::LDN;
    l.total = l.off_G + (gpre ? fct_fields<S>() * face2_geo_rows<S>(nq) * L::TE : 0);
    return l;
}

template <class S, int MINB, bool ONE = false>
__global__ void __launch_bounds__(MmaTile<S>::NT, MINB)
    face2_kernel(DevOp<double> op, FaceTiles ft, TileGeo tg, const double* __restrict__ x, double* __restrict__ y,
                 int64_t ld, int nrhs, int gpre) {
    using L = MmaTile<S>;
    using SU = Staged<S>;
    constexpr int D = S::D, NBF = S::NBF, Q = S::Q, BS = S::BS, DD = S::DD;
    constexpr int TE = L::TE, NT = L::NT, LDN = L::LDN;
    constexpr int NFLD = fct_fields<S>();
    const int nq = op.nq;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Face2Layout<S> lay = face2_layout<S>(nq, gpre);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sm = reinterpret_cast<double*>(smem_raw);
    double* TA = sm;
    double* TB = sm + lay.off_TB;
    double* Ub = sm + lay.off_U;
    double* R0 = sm + lay.off_R0;
    double* R1 = sm + lay.off_R1;
    double* Gs = sm + lay.off_G;  // the current facet tile's geometry (gpre)
    __shared__ __align__(8) unsigned long long s_gbar;
    const int nqg = face2_geo_rows<S>(nq);  // geometry rows per field
    const unsigned gbytes = static_cast<unsigned>(NFLD * nqg * TE * sizeof(double));
    if (gpre && tid == 0) mbar_init(&s_gbar, 1);
    // tile descriptors and {facet, element 0, element 1} ids of three tiles in flight: the current
    // one, the one whose blocks are being copied in, and the one after it (copied asynchronously one
    // iteration ahead, so nothing waits for them)
    __shared__ int4 s_td[3];
    __shared__ int4 s_ids[3][SU::UE];
    const int tab = lay.MF * L::LDT;
    for (int i = tid; i < 4 * SU::USZ; i += NT) Ub[i] = 0.0;

    // contiguous work ranges per CTA keep the table pair mostly unchanged
    const int64_t nwork = static_cast<int64_t>(ft.nftiles) * nrhs;
    const int64_t per = (nwork + gridDim.x - 1) / gridDim.x;
    const int64_t w0 = static_cast<int64_t>(blockIdx.x) * per;
    const int64_t w1 = (w0 + per < nwork) ? w0 + per : nwork;
    auto ids_async = [&](int64_t work, int slot) {  // the descriptor and ids of tile `work`
        int64_t t64, rhs;
        sweep_tile_rhs(work, ft.nftiles, ONE ? 1 : nrhs, t64, rhs);
        const int tile = static_cast<int>(t64);
        if (tid < TE) cp_async16(&s_ids[slot][tid], &ft.tids[static_cast<int64_t>(tile) * TE + tid]);
        if (tid == TE) cp_async16(&s_td[slot], &ft.ftiles[tile]);
    };
    auto stage = [&](int64_t work, int slot, int buf) {  // every thread; ids of `slot` visible
        int64_t t64, rhs;
        sweep_tile_rhs(work, ft.nftiles, ONE ? 1 : nrhs, t64, rhs);
        const double* xr = x + rhs * ld;
        const int4* ids = s_ids[slot];
        using SUT = Staged<S>;
        constexpr int per_el = Q * NBF;
        if constexpr (kStageByWarp) {  // one (side, element) block per warp, lanes along the block
            for (int pb = warp; pb < 2 * SUT::UE; pb += NT / 32) {
                const int side = pb / SUT::UE, te = pb % SUT::UE;
                const int e = te < TE ? (side ? ids[te].z : ids[te].y) : -1;  // warp-uniform
                if (e < 0) continue;
                double* dst = Ub + (2 * buf + side) * SUT::USZ + te * SUT::LDU;
                const double* src = xr + static_cast<int64_t>(e) * BS;
                for (int w = lane; w < per_el; w += 32) cp_async8(dst + (w / NBF) * SUT::KS + (w % NBF), src + w);
            }
        } else {
            for (int i = tid; i < 2 * SUT::UE * per_el; i += NT) {
                const int side = i / (SUT::UE * per_el), j = i % (SUT::UE * per_el);
                const int te = j / per_el, w = j % per_el;
                const int e = te < TE ? (side ? ids[te].z : ids[te].y) : -1;
                if (e >= 0)
                    cp_async8(Ub + (2 * buf + side) * SUT::USZ + te * SUT::LDU + (w / NBF) * SUT::KS + (w % NBF),
                              xr + static_cast<int64_t>(e) * BS + w);
            }
        }
    };
    int cur_a = -1, cur_b = -1;  // face tables held in TA / TB
    for (int k = 0; k < 2; ++k)
        if (w0 + k < w1) ids_async(w0 + k, k);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    if (w0 < w1) stage(w0, 0, 0);
    cp_async_commit();
    int buf = 0, slot = 0;
    for (int64_t work = w0; work < w1; ++work, buf ^= 1, slot = (slot == 2 ? 0 : slot + 1)) {
        int64_t t64, rhs;
        sweep_tile_rhs(work, ft.nftiles, ONE ? 1 : nrhs, t64, rhs);
        const int tile = static_cast<int>(t64);
        double* yr = y + rhs * ld;
        // own copies of this tile (and the next tiles' ids) landed; after the barrier everybody's
        // have, and the previous tile is done with R, the tables, the other buffer and its ids
        cp_async_wait<0>();
        __syncthreads();
        const int4 td = s_td[slot];
        const int key = td.z;
        const int l0 = key & 3, l1 = (key >> 2) & 3, mode = key >> 4;
        const bool two = (mode == 1);
        const int slot1 = slot == 2 ? 0 : slot + 1, slot2 = slot1 == 2 ? 0 : slot1 + 1;
        if (work + 1 < w1) stage(work + 1, slot1, buf ^ 1);
        if (work + 2 < w1) ids_async(work + 2, slot2);
        cp_async_commit();
        // the geometry of this tile into shared memory, behind the trace GEMMs (the previous tile's
        // pointwise phase, the last reader, ended before the barrier above)
        if (gpre && tid == 0)
            bulk_load(Gs, tg.fct + static_cast<int64_t>(tile) * NFLD * nqg * TE, gbytes, &s_gbar);
        const double* tA = kFaceTablesGlobal ? ft.tables + static_cast<int64_t>(l0) * tab : TA;
        const double* tB = kFaceTablesGlobal ? ft.tables + static_cast<int64_t>(l1) * tab : TB;
        if (!kFaceTablesGlobal && (l0 != cur_a || (two && l1 != cur_b))) {  // uniform: the key is the CTA's
            if (l0 != cur_a)
                for (int i = tid; i < tab; i += NT) TA[i] = ft.tables[static_cast<int64_t>(l0) * tab + i];
            if (two && l1 != cur_b)
                for (int i = tid; i < tab; i += NT) TB[i] = ft.tables[static_cast<int64_t>(l1) * tab + i];
            cur_a = l0;
            if (two) cur_b = l1;
            __syncthreads();
        }
        const double* U0 = Ub + (2 * buf) * SU::USZ;
        const double* U1 = Ub + (2 * buf + 1) * SU::USZ;
        const int4* sid = s_ids[slot];
        if (kGemmRows16 && lay.MF % 16 == 0) {
            if (two)
                cta_gemm_store_rows16<S, kFaceTablesGlobal>(tA, U0, R0, tB, U1, R1, lay.MF, L::KP / 4, warp, lane);
            else
                cta_gemm_store_rows16<S, kFaceTablesGlobal>(tA, U0, R0, nullptr, nullptr, nullptr, lay.MF, L::KP / 4,
                                                            warp, lane);
        } else if constexpr (kGemmRows) {
            if (two)
                cta_gemm_store_rows<S, kFaceTablesGlobal>(tA, U0, R0, tB, U1, R1, lay.MF, L::KP / 4, warp, lane);
            else
                cta_gemm_store_rows<S, kFaceTablesGlobal>(tA, U0, R0, nullptr, nullptr, nullptr, lay.MF, L::KP / 4, warp,
                                                          lane);
        } else if (two) {
            cta_gemm_store_staged<S, kFaceChains, kFaceTablesGlobal>(tA, U0, R0, tB, U1, R1, lay.MF, L::KP / 4, warp,
                                                                     lane);
        } else {
            cta_gemm_store_staged<S, kFaceChains, kFaceTablesGlobal>(tA, U0, R0, nullptr, nullptr, nullptr, lay.MF,
                                                                     L::KP / 4, warp, lane);
        }
        __syncthreads();
        const double* geo = tg.fct + static_cast<int64_t>(tile) * NFLD * nqg * TE;
        if (gpre) {
            if (!mbar_wait_bounded(&s_gbar, static_cast<unsigned>((work - w0) & 1)) && tid == 0 && tg.status)
                atomicExch(tg.status, 1);
            geo = Gs;
        }
        const double* pens = tg.pen + static_cast<int64_t>(tile) * TE;
        for (int it = tid; it < TE * nqg; it += NT) {
            const int te = it % TE, q = face2_point_swizzle<S>() ? face2_point(it / TE) : it / TE;
            if (q >= nq || sid[te].x < 0) continue;
            const double* gp = geo + it;  // field f at gp[f * nqg * TE]
            const int64_t fs = static_cast<int64_t>(nqg) * TE;
            double* ga0p = R0 + (q * D) * LDN + te * Q;
            double* gb0p = R0 + (D * nq + q) * LDN + te * Q;
            double* ga1p = R1 + (q * D) * LDN + te * Q;
            double* gb1p = R1 + (D * nq + q) * LDN + te * Q;
            double u0[Q], u1[Q], g0[D][Q], g1[D][Q];
#pragma unroll
            for (int r = 0; r < Q; ++r) {
                u0[r] = gb0p[r];
#pragma unroll
                for (int a = 0; a < D; ++a) g0[a][r] = ga0p[a * LDN + r];
                if (two) {
                    u1[r] = gb1p[r];
#pragma unroll
                    for (int a = 0; a < D; ++a) g1[a][r] = ga1p[a * LDN + r];
                } else if (mode == 3) {  // own neighbour: the other side is the element itself
                    u1[r] = u0[r];
#pragma unroll
                    for (int a = 0; a < D; ++a) g1[a][r] = g0[a][r];
                } else {
                    u1[r] = 0.0;
#pragma unroll
                    for (int a = 0; a < D; ++a) g1[a][r] = 0.0;
                }
            }
            double n[D], nu[D];
#pragma unroll
            for (int i = 0; i < D; ++i) {
                n[i] = gp[i * fs];
                nu[i] = gp[(D + i) * fs];
            }
            double Gs0[DD], Gs1[DD], cs0[DD], cs1[DD];
            if constexpr (S::KIND == kPoisson) {
#pragma unroll
                for (int c = 0; c < DD; ++c) {
                    cs0[c] = gp[(2 * D + c) * fs];
                    cs1[c] = gp[(2 * D + DD + c) * fs];
                    Gs0[c] = Gs1[c] = 0.0;
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
            const double pen = pens[te];
            const double wq = op.w[q];
            double ga[D][Q], gb[Q];
            if (mode == 2) {
                facet_lift<S, double>(2, n, nu, pen, wq, u0, g0, u1, g1, Gs0, Gs1, cs0, cs1, ga, gb);
            } else {
                double ha[D][Q], hb[Q];
                if (mode == 3)
                    facet_lift_pair<S>(n, nu, pen, wq, u0, g0, u1, g1, Gs0, Gs0, cs0, cs0, ga, gb, ha, hb);
                else
                    facet_lift_pair<S>(n, nu, pen, wq, u0, g0, u1, g1, Gs0, Gs1, cs0, cs1, ga, gb, ha, hb);
                if (two) {
#pragma unroll
                    for (int r = 0; r < Q; ++r) {
                        gb1p[r] = hb[r];
#pragma unroll
                        for (int a = 0; a < D; ++a) ga1p[a * LDN + r] = ha[a][r];
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < Q; ++r) {
                gb0p[r] = gb[r];
#pragma unroll
                for (int a = 0; a < D; ++a) ga0p[a * LDN + r] = ga[a][r];
            }
        }
        __syncthreads();
        double y0[L::YPW][2][2], y1[L::YPW][2][2];
#pragma unroll
        for (int j = 0; j < L::YPW; ++j)
#pragma unroll
            for (int a = 0; a < 2; ++a) y0[j][a][0] = y0[j][a][1] = y1[j][a][0] = y1[j][a][1] = 0.0;
        cta_gemm_acc_t_tab<L, kFaceTablesGlobal>(tA, R0, y0, lay.MF, warp, lane);
        if (two) cta_gemm_acc_t_tab<L, kFaceTablesGlobal>(tB, R1, y1, lay.MF, warp, lane);
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
                        const int4 id = sid[te];
                        if (id.x >= 0) {
                            atomicAdd(&yr[static_cast<int64_t>(id.y) * BS + k + NBF * r], y0[j][0][h] + y0[j][1][h]);
                            if (two)
                                atomicAdd(&yr[static_cast<int64_t>(id.z) * BS + k + NBF * r],
                                          y1[j][0][h] + y1[j][1][h]);
                        }
                    }
                }
            }
        }
    }
    cp_async_wait<0>();
}

}  // namespace tdg
