// p-multigrid kernels (mg.cuh).  All kernels are grid-stride loops over flat index ranges; the
// block-sparse kernels read the bs x bs column-major blocks with consecutive rows on consecutive
// threads.
#include "mg.cuh"

#include "../../../include/tandem_b200.h"

#include <algorithm>

namespace tdg {

namespace {

constexpr int kT = 256;

unsigned grid_for(int64_t n) {
    const int64_t b = (n + kT - 1) / kT;
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16)));
}

int launched() { return cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA; }

#define TDG_GRID_LOOP(g, total)                                                         \
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < (total); \
         g += static_cast<int64_t>(gridDim.x) * blockDim.x)

__global__ void __launch_bounds__(kT)
    k_probe_fill(int64_t E, const int32_t* __restrict__ colour, int c, MgInterp ip, int j0, int nj,
                 double* __restrict__ V, int64_t ld) {
    const int bsf = ip.N1 * ip.Q;
    const int64_t total = E * nj * ip.N1;  // (e, jj, k), k fastest
    TDG_GRID_LOOP(g, total) {
        const int k = static_cast<int>(g % ip.N1);
        const int jj = static_cast<int>((g / ip.N1) % nj);
        const int64_t e = g / (static_cast<int64_t>(ip.N1) * nj);
        if (colour[e] != c) continue;
        const int j = j0 + jj, p = j / ip.N2, l = j % ip.N2;
        V[jj * ld + e * bsf + p * ip.N1 + k] = ip.I[k * ip.N2 + l];
    }
}

__global__ void __launch_bounds__(kT)
    k_probe_extract(int64_t E, int NB, const int32_t* __restrict__ nbr, const int32_t* __restrict__ colour, int c,
                    MgInterp ip, int j0, int nj, const double* __restrict__ Y, int64_t ld, double* __restrict__ A) {
    const int bsf = ip.N1 * ip.Q, bsc = ip.N2 * ip.Q;
    const int64_t total = E * NB * bsc;  // (n, s, row), row fastest
    TDG_GRID_LOOP(g, total) {
        const int row = static_cast<int>(g % bsc);
        const int64_t ns = g / bsc;
        const int32_t t = nbr[ns];
        if (t < 0 || colour[t] != c) continue;
        const int64_t n = ns / NB;
        const int p = row / ip.N2, l = row % ip.N2;
        double* blk = A + ns * bsc * bsc;
        for (int jj = 0; jj < nj; ++jj) {
            const double* y = Y + jj * ld + n * bsf + p * ip.N1;
            double acc = 0.0;
            for (int k = 0; k < ip.N1; ++k) acc += ip.I[k * ip.N2 + l] * y[k];
            blk[static_cast<int64_t>(j0 + jj) * bsc + row] = acc;
        }
    }
}

// One CTA per block (n, s): T = A I in shared memory, then I^T T.
__global__ void __launch_bounds__(128)
    k_triple(int64_t E, int NB, const int32_t* __restrict__ nbr, MgInterp ip, const double* __restrict__ Af,
             double* __restrict__ Ac) {
    extern __shared__ double sm[];
    const int bsf = ip.N1 * ip.Q, bsc = ip.N2 * ip.Q;
    double* sA = sm;              // [bsf][bsf] column-major
    double* sT = sm + bsf * bsf;  // [bsc] columns of bsf rows
    for (int64_t ns = blockIdx.x; ns < E * NB; ns += gridDim.x) {
        if (nbr[ns] < 0) continue;  // uniform over the CTA
        const double* a = Af + ns * bsf * bsf;
        for (int i = threadIdx.x; i < bsf * bsf; i += blockDim.x) sA[i] = a[i];
        __syncthreads();
        for (int i = threadIdx.x; i < bsf * bsc; i += blockDim.x) {
            const int row = i % bsf, col = i / bsf;
            const int q = col / ip.N2, m = col % ip.N2;
            double acc = 0.0;
            for (int k = 0; k < ip.N1; ++k) acc += sA[(k + q * ip.N1) * bsf + row] * ip.I[k * ip.N2 + m];
            sT[col * bsf + row] = acc;
        }
        __syncthreads();
        double* out = Ac + ns * bsc * bsc;
        for (int i = threadIdx.x; i < bsc * bsc; i += blockDim.x) {
            const int row = i % bsc, col = i / bsc;
            const int p = row / ip.N2, l = row % ip.N2;
            double acc = 0.0;
            for (int k = 0; k < ip.N1; ++k) acc += ip.I[k * ip.N2 + l] * sT[col * bsf + k + p * ip.N1];
            out[col * bsc + row] = acc;
        }
        __syncthreads();
    }
}

// Column c of x, b, y starts at c * ld (nrhs columns); TA: the blocks' type (FP64, or FP32 copies
// for the mixed-precision smoother), accumulation in FP64.
template <typename TA>
__global__ void __launch_bounds__(kT)
    k_bsr_apply(int64_t E, int NB, int bs, const int32_t* __restrict__ nbr, const TA* __restrict__ A,
                const double* __restrict__ x, const double* __restrict__ b, double* __restrict__ y, int nrhs,
                int64_t ld) {
    const int64_t n = E * bs;
    TDG_GRID_LOOP(g, n * nrhs) {
        const int64_t c = g / n, gi = g % n;
        const int row = static_cast<int>(gi % bs);
        const int64_t e = gi / bs;
        const double* xc = x + c * ld;
        double acc = 0.0;
        for (int s = 0; s < NB; ++s) {
            const int32_t t = nbr[e * NB + s];
            if (t < 0) continue;
            const TA* blk = A + (e * NB + s) * bs * bs;
            const double* xt = xc + static_cast<int64_t>(t) * bs;
            for (int col = 0; col < bs; ++col) acc += static_cast<double>(blk[col * bs + row]) * xt[col];
        }
        y[c * ld + gi] = b ? b[c * ld + gi] - acc : acc;
    }
}

// The same with the block size known at compile time: the column loop unrolls, so every thread
// issues its block row's loads back to back.
template <int BS, typename TA>
__global__ void __launch_bounds__(kT)
    k_bsr_apply_t(int64_t E, int NB, const int32_t* __restrict__ nbr, const TA* __restrict__ A,
                  const double* __restrict__ x, const double* __restrict__ b, double* __restrict__ y, int nrhs,
                  int64_t ld) {
    const int64_t n = E * BS;
    TDG_GRID_LOOP(g, n * nrhs) {
        const int64_t c = g / n, gi = g % n;
        const int row = static_cast<int>(gi % BS);
        const int64_t e = gi / BS;
        const double* xc = x + c * ld;
        double acc = 0.0;
        for (int s = 0; s < NB; ++s) {
            const int32_t t = nbr[e * NB + s];
            if (t < 0) continue;
            const TA* blk = A + (e * NB + s) * (BS * BS) + row;
            const double* xt = xc + static_cast<int64_t>(t) * BS;
#pragma unroll
            for (int col = 0; col < BS; ++col) acc += static_cast<double>(blk[col * BS]) * xt[col];
        }
        y[c * ld + gi] = b ? b[c * ld + gi] - acc : acc;
    }
}

__global__ void __launch_bounds__(kT)
    k_diag_inv(int64_t E, int bs, int64_t stride, const double* __restrict__ blocks, double* __restrict__ dinv,
               int* __restrict__ status) {
    TDG_GRID_LOOP(g, E * bs) {
        const int i = static_cast<int>(g % bs);
        const int64_t e = g / bs;
        double d = blocks[e * stride + i * bs + i];
        if (!(d > 0.0)) {
            atomicExch(status, 1);
            d = 1.0;
        }
        dinv[g] = 1.0 / d;
    }
}

__global__ void __launch_bounds__(kT)
    k_self_blocks(int64_t E, int NB, int bs, const double* __restrict__ A, double* __restrict__ blk) {
    const int64_t bb = static_cast<int64_t>(bs) * bs;
    TDG_GRID_LOOP(g, E * bb) {
        const int64_t e = g / bb, i = g % bb;
        blk[g] = A[e * NB * bb + i];
    }
}

__global__ void __launch_bounds__(kT)
    k_prolong_add(int64_t E, MgInterp ip, const double* __restrict__ xc, int64_t ldc, double* __restrict__ xf,
                  int64_t ldf, int nrhs) {
    const int bsc = ip.N2 * ip.Q;
    const int64_t nf = E * ip.Q * ip.N1;
    TDG_GRID_LOOP(g, nf * nrhs) {  // gi = e * bsf + p * N1 + k
        const int64_t col = g / nf, gi = g % nf;
        const int k = static_cast<int>(gi % ip.N1);
        const int p = static_cast<int>((gi / ip.N1) % ip.Q);
        const int64_t e = gi / (static_cast<int64_t>(ip.N1) * ip.Q);
        const double* c = xc + col * ldc + e * bsc + p * ip.N2;
        double acc = 0.0;
        for (int l = 0; l < ip.N2; ++l) acc += ip.I[k * ip.N2 + l] * c[l];
        xf[col * ldf + gi] += acc;
    }
}

__global__ void __launch_bounds__(kT)
    k_restrict(int64_t E, MgInterp ip, const double* __restrict__ rf, int64_t ldf, double* __restrict__ rc,
               int64_t ldc, int nrhs) {
    const int bsf = ip.N1 * ip.Q;
    const int64_t nc = E * ip.Q * ip.N2;
    TDG_GRID_LOOP(g, nc * nrhs) {  // gi = e * bsc + p * N2 + l
        const int64_t col = g / nc, gi = g % nc;
        const int l = static_cast<int>(gi % ip.N2);
        const int p = static_cast<int>((gi / ip.N2) % ip.Q);
        const int64_t e = gi / (static_cast<int64_t>(ip.N2) * ip.Q);
        const double* f = rf + col * ldf + e * bsf + p * ip.N1;
        double acc = 0.0;
        for (int k = 0; k < ip.N1; ++k) acc += ip.I[k * ip.N2 + l] * f[k];
        rc[col * ldc + gi] = acc;
    }
}

// The P1 vectors have nrhs contiguous columns of nv * Q entries; the DG level's columns start at
// multiples of ld0.
__global__ void __launch_bounds__(kT)
    k_aux_apply(MgAux a, const double* __restrict__ x, const double* __restrict__ b, double* __restrict__ y,
                int nrhs) {
    const int Q = a.Q, QQ = a.Q * a.Q;
    const int64_t n = a.nv * Q;
    TDG_GRID_LOOP(g, n * nrhs) {
        const int64_t col = g / n, gi = g % n;
        const int64_t v = gi / Q;
        const int p = static_cast<int>(gi % Q);
        const double* xcol = x + col * n;
        double acc = 0.0;
        for (int64_t k = a.ptr[v]; k < a.ptr[v + 1]; ++k) {
            const double* blk = a.val + k * QQ + p * Q;
            const double* xw = xcol + static_cast<int64_t>(a.col[k]) * Q;
            for (int q = 0; q < Q; ++q) acc += blk[q] * xw[q];
        }
        y[g] = b ? b[g] - acc : acc;
    }
}

__global__ void __launch_bounds__(kT)
    k_aux_restrict(MgAux a, const double* __restrict__ r0, int64_t ld0, double* __restrict__ rc, int nrhs) {
    const int Q = a.Q, bs = a.Nbf * a.Q;
    const int64_t n = a.nv * Q;
    TDG_GRID_LOOP(g, n * nrhs) {
        const int64_t col = g / n, gi = g % n;
        const int64_t v = gi / Q;
        const int p = static_cast<int>(gi % Q);
        double acc = 0.0;
        for (int64_t k = a.vinc_ptr[v]; k < a.vinc_ptr[v + 1]; ++k) {
            const int32_t inc = a.vinc[k];
            const int64_t e = inc / a.NV;
            const int i = inc % a.NV;
            const double* r = r0 + col * ld0 + e * bs + p * a.Nbf;
            for (int kk = 0; kk < a.Nbf; ++kk) acc += a.T[kk * a.NV + i] * r[kk];
        }
        rc[g] = acc;
    }
}

__global__ void __launch_bounds__(kT)
    k_aux_prolong_add(MgAux a, int64_t E, const double* __restrict__ xc, double* __restrict__ x0, int64_t ld0,
                      int nrhs) {
    const int bs = a.Nbf * a.Q;
    const int64_t n0 = E * bs, nc = a.nv * a.Q;
    TDG_GRID_LOOP(g, n0 * nrhs) {  // gi = e * bs + p * Nbf + kk
        const int64_t col = g / n0, gi = g % n0;
        const int64_t e = gi / bs;
        const int p = static_cast<int>((gi % bs) / a.Nbf), kk = static_cast<int>(gi % a.Nbf);
        const double* xcol = xc + col * nc;
        double acc = 0.0;
        for (int i = 0; i < a.NV; ++i) acc += a.T[kk * a.NV + i] * xcol[static_cast<int64_t>(a.vid[e * a.NV + i]) * a.Q + p];
        x0[col * ld0 + gi] += acc;
    }
}

// Chebyshev kernels over nrhs columns of n entries at stride ld (the diagonal is shared).
__global__ void __launch_bounds__(kT)
    k_cheb_first(int64_t n, int nrhs, int64_t ld, const double* __restrict__ dinv, const double* __restrict__ r,
                 double* __restrict__ d, double* __restrict__ x, double c, int x_zero) {
    TDG_GRID_LOOP(g, n * nrhs) {
        const int64_t j = g % n, i = (g / n) * ld + j;
        const double di = c * dinv[j] * r[i];
        d[i] = di;
        x[i] = x_zero ? di : x[i] + di;
    }
}

__global__ void __launch_bounds__(kT)
    k_cheb_step(int64_t n, int nrhs, int64_t ld, const double* __restrict__ dinv, const double* __restrict__ y,
                double* __restrict__ r, double* __restrict__ d, double* __restrict__ x, double c1, double c2) {
    TDG_GRID_LOOP(g, n * nrhs) {
        const int64_t j = g % n, i = (g / n) * ld + j;
        const double ri = r[i] - y[i];
        const double di = c1 * d[i] + c2 * dinv[j] * ri;
        r[i] = ri;
        d[i] = di;
        x[i] += di;
    }
}

// y = x over nrhs columns of n entries at stride ld; y = a - y likewise.
__global__ void __launch_bounds__(kT)
    k_copy_cols(int64_t n, int nrhs, int64_t ld, const double* __restrict__ x, double* __restrict__ y) {
    TDG_GRID_LOOP(g, n * nrhs) {
        const int64_t i = (g / n) * ld + g % n;
        y[i] = x[i];
    }
}

__global__ void __launch_bounds__(kT) k_rsub_cols(int64_t n, int nrhs, int64_t ld, const double* a, double* y) {
    TDG_GRID_LOOP(g, n * nrhs) {
        const int64_t i = (g / n) * ld + g % n;
        y[i] = a[i] - y[i];
    }
}

__device__ double block_reduce(double v) {
    __shared__ double red[kT / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (wid == 0) {
        s = lane < kT / 32 ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    return s;
}

__global__ void __launch_bounds__(kT)
    k_dot_partial(int64_t n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ partial) {
    double s = 0.0;
    TDG_GRID_LOOP(i, n) s += a[i] * b[i];
    s = block_reduce(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kT) k_dot_final(const double* __restrict__ partial, double* __restrict__ out) {
    double s = 0.0;
    for (int i = threadIdx.x; i < kDotBlocks; i += kT) s += partial[i];
    s = block_reduce(s);
    if (threadIdx.x == 0) out[0] = s;
}

__global__ void __launch_bounds__(kT) k_axpby(int64_t n, double a, const double* __restrict__ x, double b, double* y) {
    TDG_GRID_LOOP(i, n) y[i] = a * x[i] + (b == 0.0 ? 0.0 : b * y[i]);
}

__global__ void __launch_bounds__(kT)
    k_mul(int64_t n, const double* __restrict__ a, const double* __restrict__ x, double* __restrict__ y) {
    TDG_GRID_LOOP(i, n) y[i] = a[i] * x[i];
}

// y may alias b (y = a - y in place)
__global__ void __launch_bounds__(kT) k_sub2(int64_t n, const double* a, const double* b, double* y) {
    TDG_GRID_LOOP(i, n) y[i] = a[i] - b[i];
}

// splitmix64 of (seed, i) -> uniform [-1, 1)
__global__ void __launch_bounds__(kT) k_random(int64_t n, uint64_t seed, double* __restrict__ y) {
    TDG_GRID_LOOP(i, n) {
        uint64_t z = seed + 0x9e3779b97f4a7c15ull * static_cast<uint64_t>(i + 1);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        y[i] = static_cast<double>(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    }
}

__global__ void __launch_bounds__(kT) k_round_to_float(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
    TDG_GRID_LOOP(i, n) b[i] = static_cast<float>(a[i]);
}

// Several right-hand sides: each thread takes one row for a group of up to RB right-hand sides
// (one accumulator each), so a block row is read from memory once per group instead of once per
// right-hand side (the level operators of a multi-RHS V-cycle, e.g. the Green's-function columns).
template <int BS, int RB, typename TA>
__global__ void __launch_bounds__(kT)
    k_bsr_apply_mr(int64_t E, int NB, const int32_t* __restrict__ nbr, const TA* __restrict__ A,
                   const double* __restrict__ x, const double* __restrict__ b, double* __restrict__ y, int nrhs,
                   int64_t ld) {
    const int64_t n = E * BS;
    const int64_t groups = (nrhs + RB - 1) / RB;
    TDG_GRID_LOOP(g, n * groups) {
        const int64_t cg = g / n, gi = g % n;
        const int64_t c0 = cg * RB;
        const int rb = static_cast<int>(nrhs - c0 < RB ? nrhs - c0 : RB);
        const int row = static_cast<int>(gi % BS);
        const int64_t e = gi / BS;
        double acc[RB];
#pragma unroll
        for (int j = 0; j < RB; ++j) acc[j] = 0.0;
        for (int s = 0; s < NB; ++s) {
            const int32_t t = nbr[e * NB + s];
            if (t < 0) continue;
            const TA* blk = A + (e * NB + s) * (BS * BS) + row;
            const double* xt = x + c0 * ld + static_cast<int64_t>(t) * BS;
#pragma unroll
            for (int col = 0; col < BS; ++col) {
                const double a = static_cast<double>(blk[col * BS]);
#pragma unroll
                for (int j = 0; j < RB; ++j)
                    if (j < rb) acc[j] += a * xt[j * ld + col];
            }
        }
#pragma unroll
        for (int j = 0; j < RB; ++j)
            if (j < rb) {
                const int64_t i = (c0 + j) * ld + gi;
                y[i] = b ? b[i] - acc[j] : acc[j];
            }
    }
}

#undef TDG_GRID_LOOP

}  // namespace

int launch_mg_probe_fill(int64_t E, const int32_t* colour, int c, MgInterp ip, int j0, int nj, double* V,
                         int64_t ld, cudaStream_t s) {
    k_probe_fill<<<grid_for(E * nj * ip.N1), kT, 0, s>>>(E, colour, c, ip, j0, nj, V, ld);
    return launched();
}

int launch_mg_probe_extract(int64_t E, int NB, const int32_t* nbr, const int32_t* colour, int c, MgInterp ip,
                            int j0, int nj, const double* Y, int64_t ld, double* A, cudaStream_t s) {
    k_probe_extract<<<grid_for(E * NB * ip.N2 * ip.Q), kT, 0, s>>>(E, NB, nbr, colour, c, ip, j0, nj, Y, ld, A);
    return launched();
}

int launch_mg_triple(int64_t E, int NB, const int32_t* nbr, MgInterp ip, const double* Af, double* Ac,
                     cudaStream_t s) {
    const int bsf = ip.N1 * ip.Q, bsc = ip.N2 * ip.Q;
    const size_t smem = sizeof(double) * (static_cast<size_t>(bsf) * bsf + static_cast<size_t>(bsf) * bsc);
    if (smem > 48 * 1024) return TDG_E_INVALID;
    const int64_t nblk = E * NB;
    k_triple<<<static_cast<unsigned>(std::min<int64_t>(nblk, 148 * 32)), 128, smem, s>>>(E, NB, nbr, ip, Af, Ac);
    return launched();
}

template <typename TA>
int launch_mg_bsr_apply(int64_t E, int NB, int bs, const int32_t* nbr, const TA* A, const double* x,
                        const double* b, double* y, int nrhs, int64_t ld, cudaStream_t s) {
    constexpr int RB = 8;
    if (nrhs > 1 && (bs == 3 || bs == 4 || bs == 6 || bs == 10 || bs == 12 || bs == 30)) {
        const unsigned gm = grid_for(E * bs * ((nrhs + RB - 1) / RB));
        switch (bs) {
#define TDG_BSR_MR_CASE(B) \
    case B: k_bsr_apply_mr<B, RB, TA><<<gm, kT, 0, s>>>(E, NB, nbr, A, x, b, y, nrhs, ld); break;
            TDG_BSR_MR_CASE(3) TDG_BSR_MR_CASE(4) TDG_BSR_MR_CASE(6) TDG_BSR_MR_CASE(10) TDG_BSR_MR_CASE(12) TDG_BSR_MR_CASE(30)
#undef TDG_BSR_MR_CASE
        }
        return launched();
    }
    const unsigned g = grid_for(E * bs * nrhs);
    switch (bs) {
#define TDG_BSR_CASE(B) \
    case B: k_bsr_apply_t<B, TA><<<g, kT, 0, s>>>(E, NB, nbr, A, x, b, y, nrhs, ld); break;
        TDG_BSR_CASE(1) TDG_BSR_CASE(2) TDG_BSR_CASE(3) TDG_BSR_CASE(4) TDG_BSR_CASE(6) TDG_BSR_CASE(10)
        TDG_BSR_CASE(12) TDG_BSR_CASE(20) TDG_BSR_CASE(30) TDG_BSR_CASE(60)
#undef TDG_BSR_CASE
        default: k_bsr_apply<TA><<<g, kT, 0, s>>>(E, NB, bs, nbr, A, x, b, y, nrhs, ld);
    }
    return launched();
}
template int launch_mg_bsr_apply<double>(int64_t, int, int, const int32_t*, const double*, const double*,
                                         const double*, double*, int, int64_t, cudaStream_t);
template int launch_mg_bsr_apply<float>(int64_t, int, int, const int32_t*, const float*, const double*,
                                        const double*, double*, int, int64_t, cudaStream_t);

int launch_round_to_float(int64_t n, const double* a, float* b, cudaStream_t s) {
    k_round_to_float<<<grid_for(n), kT, 0, s>>>(n, a, b);
    return launched();
}

int launch_mg_diag_inv(int64_t E, int bs, int64_t stride, const double* blocks, double* dinv, int* status,
                       cudaStream_t s) {
    k_diag_inv<<<grid_for(E * bs), kT, 0, s>>>(E, bs, stride, blocks, dinv, status);
    return launched();
}

int launch_mg_self_blocks(int64_t E, int NB, int bs, const double* A, double* blk, cudaStream_t s) {
    k_self_blocks<<<grid_for(E * bs * bs), kT, 0, s>>>(E, NB, bs, A, blk);
    return launched();
}

int launch_mg_prolong_add(int64_t E, MgInterp ip, const double* xc, int64_t ldc, double* xf, int64_t ldf, int nrhs,
                          cudaStream_t s) {
    k_prolong_add<<<grid_for(E * ip.Q * ip.N1 * nrhs), kT, 0, s>>>(E, ip, xc, ldc, xf, ldf, nrhs);
    return launched();
}

int launch_mg_restrict(int64_t E, MgInterp ip, const double* rf, int64_t ldf, double* rc, int64_t ldc, int nrhs,
                       cudaStream_t s) {
    k_restrict<<<grid_for(E * ip.Q * ip.N2 * nrhs), kT, 0, s>>>(E, ip, rf, ldf, rc, ldc, nrhs);
    return launched();
}

int launch_aux_apply(MgAux const& a, const double* x, const double* b, double* y, int nrhs, cudaStream_t s) {
    k_aux_apply<<<grid_for(a.nv * a.Q * nrhs), kT, 0, s>>>(a, x, b, y, nrhs);
    return launched();
}

int launch_aux_restrict(MgAux const& a, const double* r0, int64_t ld0, double* rc, int nrhs, cudaStream_t s) {
    k_aux_restrict<<<grid_for(a.nv * a.Q * nrhs), kT, 0, s>>>(a, r0, ld0, rc, nrhs);
    return launched();
}

int launch_aux_prolong_add(MgAux const& a, int64_t E, const double* xc, double* x0, int64_t ld0, int nrhs,
                           cudaStream_t s) {
    k_aux_prolong_add<<<grid_for(E * a.Nbf * a.Q * nrhs), kT, 0, s>>>(a, E, xc, x0, ld0, nrhs);
    return launched();
}

int launch_cheb_first(int64_t n, int nrhs, int64_t ld, const double* dinv, const double* r, double* d, double* x,
                      double c, int x_zero, cudaStream_t s) {
    k_cheb_first<<<grid_for(n * nrhs), kT, 0, s>>>(n, nrhs, ld, dinv, r, d, x, c, x_zero);
    return launched();
}

int launch_cheb_step(int64_t n, int nrhs, int64_t ld, const double* dinv, const double* y, double* r, double* d,
                     double* x, double c1, double c2, cudaStream_t s) {
    k_cheb_step<<<grid_for(n * nrhs), kT, 0, s>>>(n, nrhs, ld, dinv, y, r, d, x, c1, c2);
    return launched();
}

int launch_vec_copy_cols(int64_t n, int nrhs, int64_t ld, const double* x, double* y, cudaStream_t s) {
    k_copy_cols<<<grid_for(n * nrhs), kT, 0, s>>>(n, nrhs, ld, x, y);
    return launched();
}

int launch_vec_rsub_cols(int64_t n, int nrhs, int64_t ld, const double* a, double* y, cudaStream_t s) {
    k_rsub_cols<<<grid_for(n * nrhs), kT, 0, s>>>(n, nrhs, ld, a, y);
    return launched();
}

int launch_vec_dot(int64_t n, const double* a, const double* b, double* partial, double* out, cudaStream_t s) {
    k_dot_partial<<<kDotBlocks, kT, 0, s>>>(n, a, b, partial);
    k_dot_final<<<1, kT, 0, s>>>(partial, out);
    return launched();
}

int launch_vec_axpby(int64_t n, double a, const double* x, double b, double* y, cudaStream_t s) {
    k_axpby<<<grid_for(n), kT, 0, s>>>(n, a, x, b, y);
    return launched();
}

int launch_vec_mul(int64_t n, const double* a, const double* x, double* y, cudaStream_t s) {
    k_mul<<<grid_for(n), kT, 0, s>>>(n, a, x, y);
    return launched();
}

int launch_vec_sub(int64_t n, const double* a, const double* b, double* y, cudaStream_t s) {
    k_sub2<<<grid_for(n), kT, 0, s>>>(n, a, b, y);
    return launched();
}

int launch_vec_random(int64_t n, uint64_t seed, double* y, cudaStream_t s) {
    k_random<<<grid_for(n), kT, 0, s>>>(n, seed, y);
    return launched();
}

}  // namespace tdg
