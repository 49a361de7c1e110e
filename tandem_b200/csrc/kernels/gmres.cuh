// Vector kernels of the device flexible GMRES (restarted FGMRES(m), right preconditioning:
// Saad, "A flexible inner-outer preconditioned GMRES algorithm", SIAM J. Sci. Comput. 14, 1993),
// the Krylov method of tandem's multigrid configuration (examples/options/mg_cheby.cfg:
// -ksp_type fgmres).
//
// Segments and chunks as in krylov.cuh: every segment (right-hand side or independent problem)
// has its own Arnoldi process -- its own Hessenberg matrix, Givens rotations and residual estimate
// -- while every launch covers all segments.  Orthogonalisation is classical Gram-Schmidt applied
// twice (CGS2): per Arnoldi step one fused multi-dot reduction for V^T w, one update, a second
// multi-dot that also returns w.w, and a second update fused with the normalisation of the next
// basis vector; ||w - V h2||^2 = w.w - ||h2||^2 (exact for an orthonormal V, and h2 is tiny after
// the first pass, so nothing cancels).  All per-segment scalars live in device memory.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "krylov.cuh"

namespace tdg {

// per-segment state, kGm doubles per segment
constexpr int kGm = 8;
enum GmSlot { kGmBeta = 0, kGmActive = 1, kGmSteps = 2, kGmTol = 3, kGmScale = 4, kGmEst = 5 };
constexpr int kGmMaxRestart = 64;
// basis vectors handled by one multi-dot / update launch (their accumulators sit in registers)
constexpr int kGmGroup = 32;

// partial[chunk][k0 + k] = V_k . w over the chunk for k < nv, and w . w at k0 + nv when `norm`.
// V_k = V + k * vstride.
template <int MAXV>
__global__ void __launch_bounds__(kVecThreads)
    k_gm_dots(const Chunk* __restrict__ chunks, const double* __restrict__ V, int64_t vstride, int nv,
              const double* __restrict__ w, int norm, double* __restrict__ partial, int pstride, int k0) {
    const Chunk ch = chunks[blockIdx.x];
    double acc[MAXV + 1];
#pragma unroll
    for (int k = 0; k <= MAXV; ++k) acc[k] = 0.0;
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        const double wv = w[i];
#pragma unroll
        for (int k = 0; k < MAXV; ++k)
            if (k < nv) acc[k] = fma(V[k * vstride + i], wv, acc[k]);
        acc[MAXV] = fma(wv, wv, acc[MAXV]);
    }
    __shared__ double red[MAXV + 1][kVecThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k <= MAXV; ++k) {
        if (k < nv || k == MAXV) {
            const double v = warp_sum(acc[k]);
            if (lane == 0) red[k][wid] = v;
        }
    }
    __syncthreads();
    const int nout = nv + (norm ? 1 : 0);
    for (int k = threadIdx.x; k < nout; k += blockDim.x) {
        const int src = k < nv ? k : MAXV;
        double s = 0.0;
        for (int q = 0; q < kVecThreads / 32; ++q) s += red[src][q];
        partial[static_cast<int64_t>(blockIdx.x) * pstride + k0 + k] = s;
    }
}

// out[seg][k] = sum of the segment's chunk partials, k < nout.
__global__ void k_gm_reduce(const double* __restrict__ partial, int pstride, const int* __restrict__ seg_chunk,
                            int nout, double* __restrict__ out, int ostride) {
    const int seg = blockIdx.x;
    for (int k = threadIdx.x; k < nout; k += blockDim.x) {
        double s = 0.0;
        for (int c = seg_chunk[seg]; c < seg_chunk[seg + 1]; ++c) s += partial[static_cast<int64_t>(c) * pstride + k];
        out[static_cast<int64_t>(seg) * ostride + k] = s;
    }
}

// w -= sum_{k < nv} V_k coef[seg][k]; with `out`: out = scale[seg] * (w - ...), w untouched.
// Inactive segments: w unchanged, out = 0.
template <int MAXV>
__global__ void __launch_bounds__(kVecThreads)
    k_gm_update(const Chunk* __restrict__ chunks, const double* __restrict__ V, int64_t vstride, int nv,
                double* __restrict__ w, const double* __restrict__ coef, int cstride, const double* __restrict__ st,
                double* __restrict__ out) {
    const Chunk ch = chunks[blockIdx.x];
    const double* sg = st + ch.seg * kGm;
    const bool active = sg[kGmActive] != 0.0;
    __shared__ double c[MAXV];
    for (int k = threadIdx.x; k < nv; k += blockDim.x) c[k] = coef[static_cast<int64_t>(ch.seg) * cstride + k];
    __syncthreads();
    if (!active) {
        if (out)
            for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) out[i] = 0.0;
        return;
    }
    const double scale = out ? sg[kGmScale] : 1.0;
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        double v = w[i];
#pragma unroll
        for (int k = 0; k < MAXV; ++k)
            if (k < nv) v = fma(-V[k * vstride + i], c[k], v);
        if (out)
            out[i] = scale * v;
        else
            w[i] = v;
    }
}

// First Gram-Schmidt pass of Arnoldi step j: H[:, j] = h1 (the reduced dots) for active segments.
// H per segment column-major [(m + 1) x m], leading dimension m + 1.
__global__ void k_gm_pass1(const double* __restrict__ h1, int hstride, double* __restrict__ H, int m, int j, int nseg,
                           const double* __restrict__ st) {
    const int seg = blockIdx.x;
    if (seg >= nseg) return;
    const bool active = st[seg * kGm + kGmActive] != 0.0;
    double* Hc = H + static_cast<int64_t>(seg) * (m + 1) * m + static_cast<int64_t>(j) * (m + 1);
    for (int k = threadIdx.x; k <= j; k += blockDim.x) Hc[k] = active ? h1[static_cast<int64_t>(seg) * hstride + k] : 0.0;
}

// Second pass of step j, one thread per segment: H[:, j] += h2, H[j+1][j] = ||w|| after the
// second update (w.w - ||h2||^2), the previous Givens rotations applied to column j and a new one
// computed; g (the rotated right-hand side beta e_1) updated, the residual estimate |g[j+1]|.
// A segment whose estimate meets its tolerance, or whose new basis vector vanishes (the Krylov
// space holds the solution), stops taking steps.  kGmScale = 1 / H[j+1][j] for the next basis
// vector (0 when stopped).
__global__ void k_gm_pass2(const double* __restrict__ h2, int hstride, double* __restrict__ H, double* __restrict__ cs,
                           double* __restrict__ sn, double* __restrict__ g, int m, int j, int nseg,
                           double* __restrict__ st) {
    const int seg = blockIdx.x * blockDim.x + threadIdx.x;
    if (seg >= nseg) return;
    double* sg = st + seg * kGm;
    sg[kGmScale] = 0.0;
    if (sg[kGmActive] == 0.0) return;
    double* Hc = H + static_cast<int64_t>(seg) * (m + 1) * m + static_cast<int64_t>(j) * (m + 1);
    double* c = cs + static_cast<int64_t>(seg) * m;
    double* s = sn + static_cast<int64_t>(seg) * m;
    double* gg = g + static_cast<int64_t>(seg) * (m + 1);
    const double* hh = h2 + static_cast<int64_t>(seg) * hstride;
    double h2sq = 0.0, colsq = 0.0;
    for (int k = 0; k <= j; ++k) {
        Hc[k] += hh[k];
        h2sq += hh[k] * hh[k];
        colsq += Hc[k] * Hc[k];
    }
    const double ww = hh[j + 1];  // w.w before the second update
    const double hn = sqrt(fmax(ww - h2sq, 0.0));
    Hc[j + 1] = hn;
    for (int k = 0; k < j; ++k) {
        const double a = Hc[k], b = Hc[k + 1];
        Hc[k] = c[k] * a + s[k] * b;
        Hc[k + 1] = -s[k] * a + c[k] * b;
    }
    const double a = Hc[j], b = Hc[j + 1];
    const double r = hypot(a, b);
    const double cj = r > 0.0 ? a / r : 1.0, sj = r > 0.0 ? b / r : 0.0;
    c[j] = cj;
    s[j] = sj;
    Hc[j] = r;
    Hc[j + 1] = 0.0;
    gg[j + 1] = -sj * gg[j];
    gg[j] = cj * gg[j];
    const double est = fabs(gg[j + 1]);
    sg[kGmSteps] = j + 1;
    sg[kGmEst] = est;
    const bool breakdown = !(hn > 1e-14 * sqrt(colsq + hn * hn));
    if (est <= sg[kGmTol] || breakdown || !(est == est) || r == 0.0)
        sg[kGmActive] = 0.0;
    else
        sg[kGmScale] = 1.0 / hn;
}

// v0 = r / beta on active segments, 0 elsewhere.
__global__ void __launch_bounds__(kVecThreads)
    k_gm_start(const Chunk* __restrict__ chunks, const double* __restrict__ r, double* __restrict__ v0,
               const double* __restrict__ st) {
    const Chunk ch = chunks[blockIdx.x];
    const double* sg = st + ch.seg * kGm;
    const double sc = (sg[kGmActive] != 0.0 && sg[kGmBeta] > 0.0) ? 1.0 / sg[kGmBeta] : 0.0;
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) v0[i] = sc * r[i];
}

// y = R^-1 g over the segment's steps (R the rotated Hessenberg matrix, upper triangular), one
// thread per segment; y [nseg][m], zero beyond the segment's steps.
__global__ void k_gm_solve_y(const double* __restrict__ H, const double* __restrict__ g, double* __restrict__ y, int m,
                             int nseg, const double* __restrict__ st) {
    const int seg = blockIdx.x * blockDim.x + threadIdx.x;
    if (seg >= nseg) return;
    const int ks = static_cast<int>(st[seg * kGm + kGmSteps]);
    const double* Hs = H + static_cast<int64_t>(seg) * (m + 1) * m;
    const double* gg = g + static_cast<int64_t>(seg) * (m + 1);
    double* ys = y + static_cast<int64_t>(seg) * m;
    for (int k = ks; k < m; ++k) ys[k] = 0.0;
    for (int k = ks - 1; k >= 0; --k) {
        double v = gg[k];
        for (int q = k + 1; q < ks; ++q) v -= Hs[k + static_cast<int64_t>(q) * (m + 1)] * ys[q];
        const double d = Hs[k + static_cast<int64_t>(k) * (m + 1)];
        ys[k] = d != 0.0 ? v / d : 0.0;
    }
}

// x += sum_k Z_k y[seg][k] (Z_k = Z + k * vstride, k < nv; y zero beyond each segment's steps).
template <int MAXV>
__global__ void __launch_bounds__(kVecThreads)
    k_gm_update_x(const Chunk* __restrict__ chunks, const double* __restrict__ Z, int64_t vstride, int nv,
                  double* __restrict__ x, const double* __restrict__ y, int m) {
    const Chunk ch = chunks[blockIdx.x];
    __shared__ double c[MAXV];
    for (int k = threadIdx.x; k < nv; k += blockDim.x) c[k] = y[static_cast<int64_t>(ch.seg) * m + k];
    __syncthreads();
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        double v = x[i];
#pragma unroll
        for (int k = 0; k < MAXV; ++k)
            if (k < nv) v = fma(Z[k * vstride + i], c[k], v);
        x[i] = v;
    }
}

}  // namespace tdg
