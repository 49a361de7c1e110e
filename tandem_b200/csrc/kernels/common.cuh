// Shared device-side definitions: operator parameter block and compile-time sizes.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tdg {

constexpr int kPoisson = 0;
constexpr int kElasticity = 1;

__host__ __device__ constexpr int cbinom(int n, int k) {
    int r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

// ---- work items --------------------------------------------------------------------------------------

// Work item -> (tile, right-hand side) of a multi-RHS apply.  Items run over groups of kRhsGroup
// right-hand sides; inside a group the tile is the slower index and the right-hand side the faster
// one, so consecutive items (a CTA's own, and those the CTAs run at one time) read the same tile's
// geometry: it comes from memory once per group and then from L2, while a group's vectors
// (kRhsGroup x the vector) stay small enough to be reused from L2 as well.  One right-hand side:
// item = tile.
constexpr int kRhsGroup = 8;
__device__ __forceinline__ void work_tile_rhs(int64_t work, int64_t ntiles, int nrhs, int64_t& tile, int64_t& rhs) {
    // the kernels that call this per tile are issue-bound: one right-hand side needs no division,
    // and 32-bit division serves every item count below 2^32
    if (nrhs == 1) {
        tile = work;
        rhs = 0;
        return;
    }
    const int64_t full = nrhs / kRhsGroup;  // complete groups
    const int64_t per = ntiles * kRhsGroup;
    if (static_cast<uint64_t>(ntiles) * static_cast<uint64_t>(nrhs) <= 0xffffffffull) {
        const uint32_t w32 = static_cast<uint32_t>(work), per32 = static_cast<uint32_t>(per);
        const uint32_t full32 = static_cast<uint32_t>(full);
        if (w32 < full32 * per32) {
            const uint32_t grp = w32 / per32, w = w32 - grp * per32;
            tile = w / kRhsGroup;
            rhs = static_cast<int64_t>(grp) * kRhsGroup + (w % kRhsGroup);
        } else {
            const uint32_t w = w32 - full32 * per32, rest = static_cast<uint32_t>(nrhs) - full32 * kRhsGroup;
            const uint32_t t = w / rest;
            tile = t;
            rhs = static_cast<int64_t>(full32) * kRhsGroup + (w - t * rest);
        }
        return;
    }
    if (work < full * per) {
        const int64_t grp = work / per, w = work - grp * per;
        tile = w / kRhsGroup;
        rhs = grp * kRhsGroup + (w - tile * kRhsGroup);
    } else {  // the last, partial group of `rest` right-hand sides
        const int64_t w = work - full * per;
        const int64_t rest = nrhs - full * kRhsGroup;
        tile = w / rest;
        rhs = full * kRhsGroup + (w - tile * rest);
    }
}

// Compile-time shape of one (dimension, degree, operator) instance.
template <int D_, int N_, int KIND_>
struct Shape {
    static constexpr int D = D_;
    static constexpr int N = N_;
    static constexpr int KIND = KIND_;
    static constexpr int NBF = cbinom(N_ + D_, D_);
    static constexpr int Q = (KIND_ == kPoisson) ? 1 : D_;
    static constexpr int BS = NBF * Q;
    static constexpr int DD = D_ * D_;
    static constexpr int NF = D_ + 1;
};

// Device-resident operator data in one precision T (see host/setup.hpp for the meaning of each
// array; the device copies keep the same index order, plus transposed basis tables so that
// threads indexed by basis function read contiguous memory).
template <typename T>
struct DevOp {
    int64_t E = 0, F = 0;
    int Nq = 0, nq = 0;
    const T* Dxi_Q = nullptr;   // [NBF][D][Nq]
    const T* DxiT_Q = nullptr;  // [D][Nq][NBF]
    const T* E_q = nullptr;     // [NF][NBF][nq]
    const T* ET_q = nullptr;    // [NF][nq][NBF]
    const T* Dxi_q = nullptr;   // [NF][NBF][D][nq]
    const T* DxiT_q = nullptr;  // [NF][D][nq][NBF]
    const T* w = nullptr;       // [nq]
    const T* vG = nullptr;      // [E][DD][Nq]
    const T* vCoef = nullptr;   // [E][ncoef][Nq]
    const T* fN = nullptr;      // [F][D][nq]
    const T* fNunit = nullptr;  // [F][D][nq]
    const T* fNl = nullptr;     // [F][nq]
    const T* fCoef = nullptr;   // Poisson [F][2][DD][nq] (K G0, K G1); Elasticity [F][4][nq]
    const T* fG = nullptr;      // [F][2][DD][nq] (G0, G1)
    const double* penalty = nullptr;  // [F], kept in FP64 for every precision
    const int4* sides = nullptr;      // [E][NF] {fct, side | bc << 8, nb, nb_local}
};

}  // namespace tdg
