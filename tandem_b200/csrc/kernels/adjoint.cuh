// Gradient of a functional J(u(theta)) with respect to per-element constant Lame parameters
// theta_e = (lambda_e, mu_e) of the elasticity operator, from the state u and the adjoint p
// (A p = dJ/du; the SIPG operator is symmetric, so the adjoint solve reuses A):
//
//   dJ/dtheta_e = p^T db/dtheta_e - p^T (dA/dtheta_e) u.
//
// A depends on theta_e through the volume coefficients lam W |J|, mu W |J| of element e
// (apply_volume, app/kernels/elasticity.py:224-229), the facet coefficients lam_q, mu_q of the
// sides that belong to e (flux_sigma_* and apply_facet, elasticity.py:201-234, with tandem's side
// swap, Elasticity.cpp:734-747), and the interior penalty of the facets of e
// (Elasticity::prepare_penalty, Elasticity.cpp:279-292: p_s = (D+1) c_{N-1} |f|/|E_s| c1^2/c0,
// c0 = min 2 mu, c1 = max(D lam + 2 mu); interior (p0 + p1)/4).  b depends on theta_e through the
// Dirichlet lift on the boundary facets (rhs_boundary / rhs_skeleton, elasticity.py:154-179).
//
// Contracting the element-centric apply with p gives, per facet side o with outward normal n_o,
// jumps [u] = u_o - u_n, [p] = p_o - p_n (interior, factor 1/2) or [u] = u_o, [p] = p_o
// (Dirichlet / fault boundary, factor 1):
//   dlam_o: -f sum_q w (div p_o [u].n + div u_o [p].n)
//   dmu_o : -f sum_q w ([u].(grad p_o + grad p_o^T) n + [p].(grad u_o + grad u_o^T) n)
//   pen   : dpen/dtheta_o sum_q w |n| [p].[u]
// and for the volume dlam = sum_q W|J| div u div p, dmu = sum_q W|J| (grad u + grad u^T):grad p.
// One CTA per element; every term above is symmetric in (u, p), as it must be for symmetric A.
#pragma once

#include "common.cuh"

namespace tdg {

constexpr int kAdjThreads = 64;

template <class S>
__global__ void __launch_bounds__(kAdjThreads)
    adjoint_lame_kernel(DevOp<double> op, const double* __restrict__ u, const double* __restrict__ p,
                        const double* __restrict__ bcq, const double* __restrict__ dpen, double* __restrict__ grad) {
    constexpr int D = S::D, NBF = S::NBF, BS = S::BS, DD = S::DD, NF = S::NF;
    static_assert(S::KIND == kElasticity, "Lame gradient of the elasticity operator");
    const int Nq = op.Nq, nq = op.nq;
    const int64_t e = blockIdx.x;
    const int tid = threadIdx.x;
    __shared__ double su[BS], sp[BS], sun[BS], spn[BS];
    __shared__ double red[2][kAdjThreads / 32];
    for (int i = tid; i < BS; i += blockDim.x) {
        su[i] = u[e * BS + i];
        sp[i] = p[e * BS + i];
    }
    __syncthreads();
    double gl = 0.0, gm = 0.0;  // p^T db - p^T dA u accumulated per thread

    // volume
    for (int q = tid; q < Nq; q += blockDim.x) {
        double G[DD];
#pragma unroll
        for (int c = 0; c < DD; ++c) G[c] = op.vG[(e * DD + c) * Nq + q];
        double ru[D][D], rp[D][D];  // reference gradients [a][r]
#pragma unroll
        for (int a = 0; a < D; ++a)
#pragma unroll
            for (int r = 0; r < D; ++r) ru[a][r] = rp[a][r] = 0.0;
        for (int k = 0; k < NBF; ++k)
#pragma unroll
            for (int a = 0; a < D; ++a) {
                const double dv = op.Dxi_Q[(k * D + a) * Nq + q];
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    ru[a][r] += dv * su[k + NBF * r];
                    rp[a][r] += dv * sp[k + NBF * r];
                }
            }
        // physical gradients Ju[r][s] = d u_r / d x_s
        double Ju[D][D], Jp[D][D];
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int s = 0; s < D; ++s) {
                double a0 = 0.0, a1 = 0.0;
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    a0 += G[a * D + s] * ru[a][r];
                    a1 += G[a * D + s] * rp[a][r];
                }
                Ju[r][s] = a0;
                Jp[r][s] = a1;
            }
        double du = 0.0, dp = 0.0, sym = 0.0;
#pragma unroll
        for (int r = 0; r < D; ++r) {
            du += Ju[r][r];
            dp += Jp[r][r];
#pragma unroll
            for (int s = 0; s < D; ++s) sym += (Ju[r][s] + Ju[s][r]) * Jp[r][s];
        }
        // vCoef holds lam W |J| and mu W |J|; W |J| is recovered from the lambda coefficient of a
        // constant field: W |J| = lam W |J| / lam_e.  The host passes lam_e, mu_e through dpen.
        const double lamWJ = op.vCoef[(e * 2 + 0) * Nq + q];
        const double wj = lamWJ / dpen[static_cast<int64_t>(op.F) * 4 + 2 * e];
        gl -= wj * du * dp;
        gm -= wj * sym;
    }

    // facets
    for (int f = 0; f < NF; ++f) {
        const int4 sd = op.sides[e * NF + f];
        const int bcv = sd.y >> 8;
        const bool skel = sd.z != static_cast<int>(e);
        const bool fd = (bcv == 3 || bcv == 5);
        const int mode = (bcv == 0 || (skel && fd)) ? 1 : (fd ? 2 : 0);
        __syncthreads();
        if (mode == 1)
            for (int i = tid; i < BS; i += blockDim.x) {
                sun[i] = u[static_cast<int64_t>(sd.z) * BS + i];
                spn[i] = p[static_cast<int64_t>(sd.z) * BS + i];
            }
        __syncthreads();
        if (mode == 0) continue;
        const int fct = sd.x;
        const int side = sd.y & 0xff;
        const int own = skel ? side : 0;
        const double flip = (skel && side == 1) ? -1.0 : 1.0;
        const double fac = (mode == 1) ? 0.5 : 1.0;
        const double dpl = dpen[static_cast<int64_t>(fct) * 4 + 2 * own + 0];
        const double dpm = dpen[static_cast<int64_t>(fct) * 4 + 2 * own + 1];
        const int nbl = sd.w;
        for (int q = tid; q < nq; q += blockDim.x) {
            double G[DD];
#pragma unroll
            for (int c = 0; c < DD; ++c) G[c] = op.fG[((static_cast<int64_t>(fct) * 2 + own) * DD + c) * nq + q];
            double tu[D], tp[D], ru[D][D], rp[D][D], tun[D], tpn[D];
#pragma unroll
            for (int r = 0; r < D; ++r) {
                tu[r] = tp[r] = tun[r] = tpn[r] = 0.0;
#pragma unroll
                for (int a = 0; a < D; ++a) ru[a][r] = rp[a][r] = 0.0;
            }
            for (int k = 0; k < NBF; ++k) {
                const double ev = op.E_q[(f * NBF + k) * nq + q];
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    tu[r] += ev * su[k + NBF * r];
                    tp[r] += ev * sp[k + NBF * r];
                }
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    const double dv = op.Dxi_q[((f * NBF + k) * D + a) * nq + q];
#pragma unroll
                    for (int r = 0; r < D; ++r) {
                        ru[a][r] += dv * su[k + NBF * r];
                        rp[a][r] += dv * sp[k + NBF * r];
                    }
                }
                if (mode == 1) {
                    const double en = op.E_q[(nbl * NBF + k) * nq + q];
#pragma unroll
                    for (int r = 0; r < D; ++r) {
                        tun[r] += en * sun[k + NBF * r];
                        tpn[r] += en * spn[k + NBF * r];
                    }
                }
            }
            double Ju[D][D], Jp[D][D];
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int s = 0; s < D; ++s) {
                    double a0 = 0.0, a1 = 0.0;
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        a0 += G[a * D + s] * ru[a][r];
                        a1 += G[a * D + s] * rp[a][r];
                    }
                    Ju[r][s] = a0;
                    Jp[r][s] = a1;
                }
            double n[D], nl2 = 0.0;
#pragma unroll
            for (int i = 0; i < D; ++i) {
                n[i] = flip * op.fN[(static_cast<int64_t>(fct) * D + i) * nq + q];
                nl2 += n[i] * n[i];
            }
            const double nl = sqrt(nl2);
            const double wq = op.w[q];
            double ju[D], jp[D];
#pragma unroll
            for (int r = 0; r < D; ++r) {
                ju[r] = tu[r] - tun[r];
                jp[r] = tp[r] - tpn[r];
            }
            double du = 0.0, dp = 0.0, jun = 0.0, jpn = 0.0, su_ = 0.0, sp_ = 0.0, pen_jj = 0.0;
#pragma unroll
            for (int r = 0; r < D; ++r) {
                du += Ju[r][r];
                dp += Jp[r][r];
                jun += ju[r] * n[r];
                jpn += jp[r] * n[r];
                pen_jj += jp[r] * ju[r];
#pragma unroll
                for (int s = 0; s < D; ++s) {
                    su_ += ju[r] * (Jp[r][s] + Jp[s][r]) * n[s];
                    sp_ += jp[r] * (Ju[r][s] + Ju[s][r]) * n[s];
                }
            }
            // operator part (subtracted): facet coefficient terms and the penalty
            gl -= wq * (-fac * (dp * jun + du * jpn) + dpl * nl * pen_jj);
            gm -= wq * (-fac * (su_ + sp_) + dpm * nl * pen_jj);
            // right-hand side part: Dirichlet / slip data g on Dirichlet and fault facets
            // (rhs_boundary / rhs_skeleton): b_s += c10 sum w sigma_s(phi) n.g + c20_s sum w |n| phi.g
            // with c20 = +pen (side 0) / -pen (side 1); the penalty depends on both sides, so its
            // derivative multiplies the jump of the adjoint trace.
            if (bcq && fd) {
                double g[D], gn = 0.0, gsym = 0.0, pg = 0.0;
                const bool boundary = !skel;
                const double half = (boundary && bcv == 3) ? 0.5 : 1.0;  // bc_boundary halves slip
#pragma unroll
                for (int i = 0; i < D; ++i) g[i] = half * bcq[(static_cast<int64_t>(fct) * D + i) * nq + q];
                // g and the normal of the lift are those of side 0
                double n0[D];
#pragma unroll
                for (int i = 0; i < D; ++i) n0[i] = op.fN[(static_cast<int64_t>(fct) * D + i) * nq + q];
                const double sg = (boundary || side == 0) ? 1.0 : -1.0;
#pragma unroll
                for (int i = 0; i < D; ++i) {
                    gn += g[i] * n0[i];
                    pg += sg * (tp[i] - tpn[i]) * g[i];  // side-0 trace minus side-1 trace
#pragma unroll
                    for (int s2 = 0; s2 < D; ++s2) gsym += g[i] * (Jp[i][s2] + Jp[s2][i]) * n0[s2];
                }
                const double c10 = boundary ? -1.0 : -0.5;
                gl += wq * (c10 * dp * gn + dpl * nl * pg);
                gm += wq * (c10 * gsym + dpm * nl * pg);
            }
        }
    }
    // block reduction
    for (int o = 16; o > 0; o >>= 1) {
        gl += __shfl_xor_sync(0xffffffffu, gl, o);
        gm += __shfl_xor_sync(0xffffffffu, gm, o);
    }
    __syncthreads();
    if ((tid & 31) == 0) {
        red[0][tid >> 5] = gl;
        red[1][tid >> 5] = gm;
    }
    __syncthreads();
    if (tid == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < kAdjThreads / 32; ++w) {
            a += red[0][w];
            b += red[1][w];
        }
        grad[2 * e] = a;
        grad[2 * e + 1] = b;
    }
}

}  // namespace tdg
