// Matrix-free SIPG operator apply y = A x on the device.
//
// One CTA processes a tile of TE elements for one right-hand side and owns the tile's output
// block in registers (thread t holds output entries t, t + NT, ...).  For each tile:
//   1. volume: reference gradients of u at the volume points (contraction with Dxi_Q), the
//      pointwise flux (Poisson: J W K grad u; Elasticity: the Lame stress lam W J tr(eps) I +
//      2 mu W J eps), mapped back with G, and the transposed contraction into the output
//      (tandem kernels apply_volume, app/kernels/poisson.py:133-136, elasticity.py:224-229);
//   2. per local face: traces of the element and of its face neighbour at the facet points,
//      the numerical fluxes u_hat - u and sigma_hat (flux_u_* / flux_sigma_*, poisson.py:123-132,
//      elasticity.py:201-220) and the lift-back (apply_facet, poisson.py:137-140,
//      elasticity.py:230-234), with tandem's side-1 convention (normals negated, side data
//      swapped; Poisson.cpp:576-587, Elasticity.cpp:734-747) and its BC branching
//      (Poisson.cpp:591-631).
// The element-centric form evaluates every interior facet from both sides, as tandem's
// DGOperator::apply_ does (src/form/DGOperator.h:363-396); it needs no atomics and writes each
// output block exactly once.
#pragma once

#include "common.cuh"

namespace tdg {

template <class S>
struct ApplyTile {
    static constexpr int NT = 256;
    static constexpr int TE0 = 1024 / S::BS;
    static constexpr int TE = TE0 < 1 ? 1 : (TE0 > 64 ? 64 : TE0);
    static constexpr int ITEMS = (TE * S::BS + NT - 1) / NT;
};

template <class S, typename T>
__host__ __device__ inline int apply_smem_elems(int Nq, int nq) {
    using Tl = ApplyTile<S>;
    int vol = Tl::TE * S::Q * S::D * Nq;
    int fct = Tl::TE * S::Q * (S::D + 1) * nq;
    return 2 * Tl::TE * S::BS + (vol > fct ? vol : fct);
}

template <class S, typename T>
__global__ void __launch_bounds__(ApplyTile<S>::NT)
    apply_kernel(DevOp<T> op, const T* __restrict__ x, T* __restrict__ y, int64_t ld) {
    using Tl = ApplyTile<S>;
    constexpr int D = S::D, NBF = S::NBF, Q = S::Q, BS = S::BS, DD = S::DD, NF = S::NF;
    constexpr int TE = Tl::TE, NT = Tl::NT, ITEMS = Tl::ITEMS;
    const int Nq = op.Nq, nq = op.nq;
    const int64_t E = op.E;
    const int tid = threadIdx.x;
    const int rhs = blockIdx.y;
    x += rhs * ld;
    y += rhs * ld;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sU = reinterpret_cast<T*>(smem_raw);
    T* sUn = sU + TE * BS;
    T* sT = sUn + TE * BS;  // volume stresses, then facet lift inputs (A then B)

    const int64_t ntiles = (E + TE - 1) / TE;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t e0 = tile * TE;
        __syncthreads();
        for (int i = tid; i < TE * BS; i += NT) {
            int64_t e = e0 + i / BS;
            sU[i] = (e < E) ? x[e0 * BS + i] : T(0);
        }
        __syncthreads();

        // ---- volume: pointwise stresses at (element, point) items ----
        for (int it = tid; it < TE * Nq; it += NT) {
            const int te = it / Nq, q = it - te * Nq;
            const int64_t e = e0 + te;
            if (e >= E) continue;
            T gr[D][Q];
#pragma unroll
            for (int a = 0; a < D; ++a)
#pragma unroll
                for (int r = 0; r < Q; ++r) gr[a][r] = T(0);
            const T* u = sU + te * BS;
            for (int k = 0; k < NBF; ++k) {
                T uk[Q];
#pragma unroll
                for (int r = 0; r < Q; ++r) uk[r] = u[k + NBF * r];
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    T dv = __ldg(&op.Dxi_Q[(k * D + a) * Nq + q]);
#pragma unroll
                    for (int r = 0; r < Q; ++r) gr[a][r] += dv * uk[r];
                }
            }
            T G[DD];
            const T* vg = op.vG + e * DD * Nq + q;
#pragma unroll
            for (int c = 0; c < DD; ++c) G[c] = vg[c * Nq];
            T* st = sT + te * Q * D * Nq + q;
            if constexpr (S::KIND == kPoisson) {
                const T jwk = op.vCoef[e * Nq + q];
                T gx[D];
#pragma unroll
                for (int i = 0; i < D; ++i) {
                    T s = T(0);
#pragma unroll
                    for (int a = 0; a < D; ++a) s += G[a * D + i] * gr[a][0];
                    gx[i] = jwk * s;
                }
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    T s = T(0);
#pragma unroll
                    for (int i = 0; i < D; ++i) s += G[a * D + i] * gx[i];
                    st[a * Nq] = s;
                }
            } else {
                const T lam = op.vCoef[(e * 2 + 0) * Nq + q];
                const T mu = op.vCoef[(e * 2 + 1) * Nq + q];
                // Ju[s][r] = d u_r / d x_s
                T Ju[D][D];
#pragma unroll
                for (int s = 0; s < D; ++s)
#pragma unroll
                    for (int r = 0; r < D; ++r) {
                        T acc = T(0);
#pragma unroll
                        for (int a = 0; a < D; ++a) acc += G[a * D + s] * gr[a][r];
                        Ju[s][r] = acc;
                    }
                T div = T(0);
#pragma unroll
                for (int r = 0; r < D; ++r) div += Ju[r][r];
#pragma unroll
                for (int uu = 0; uu < D; ++uu) {
                    T sig[D];
#pragma unroll
                    for (int j = 0; j < D; ++j)
                        sig[j] = mu * (Ju[uu][j] + Ju[j][uu]) + ((uu == j) ? lam * div : T(0));
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        T s = T(0);
#pragma unroll
                        for (int j = 0; j < D; ++j) s += G[a * D + j] * sig[j];
                        st[(uu * D + a) * Nq] = s;
                    }
                }
            }
        }
        __syncthreads();

        // ---- volume: transposed contraction into the register-resident output ----
        T acc[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            acc[j] = T(0);
            const int it = tid + j * NT;
            if (it < TE * BS) {
                const int te = it / BS, rem = it - te * BS;
                const int uu = rem / NBF, k = rem - uu * NBF;
                const T* st = sT + (te * Q + uu) * D * Nq;
                T s = T(0);
                for (int c = 0; c < D * Nq; ++c) s += __ldg(&op.DxiT_Q[c * NBF + k]) * st[c];
                acc[j] = s;
            }
        }

        // ---- facets ----
        for (int f = 0; f < NF; ++f) {
            __syncthreads();
            for (int i = tid; i < TE * BS; i += NT) {
                const int te = i / BS;
                const int64_t e = e0 + te;
                T v = T(0);
                if (e < E) {
                    const int nb = op.sides[e * NF + f].z;
                    v = x[static_cast<int64_t>(nb) * BS + (i - te * BS)];
                }
                sUn[i] = v;
            }
            __syncthreads();
            T* sA = sT;                       // [TE][Q][D][nq]
            T* sB = sT + TE * Q * D * nq;     // [TE][Q][nq]
            for (int it = tid; it < TE * nq; it += NT) {
                const int te = it / nq, q = it - te * nq;
                const int64_t e = e0 + te;
                T* a_out = sA + te * Q * D * nq + q;
                T* b_out = sB + te * Q * nq + q;
                int mode = 0;  // 0 skip, 1 skeleton, 2 boundary
                int4 sd = make_int4(0, 0, 0, 0);
                if (e < E) {
                    sd = op.sides[e * NF + f];
                    const int bcv = sd.y >> 8;
                    const bool skel = sd.z != static_cast<int>(e);
                    const bool fd = (bcv == 3 || bcv == 5);
                    mode = (bcv == 0 || (skel && fd)) ? 1 : (fd ? 2 : 0);
                }
                if (mode == 0) {
#pragma unroll
                    for (int c = 0; c < Q * D; ++c) a_out[c * nq] = T(0);
#pragma unroll
                    for (int c = 0; c < Q; ++c) b_out[c * nq] = T(0);
                    continue;
                }
                const int fct = sd.x;
                const int side = sd.y & 0xff;
                const bool skel = sd.z != static_cast<int>(e);
                const int nbl = sd.w;
                const int own = skel ? side : 0;
                const int oth = skel ? 1 - side : 0;
                const T flip = (skel && side == 1) ? T(-1) : T(1);

                // traces: u and reference gradients, own side (face f) and neighbour (face nbl)
                T u0[Q], u1[Q], g0[D][Q], g1[D][Q];
#pragma unroll
                for (int r = 0; r < Q; ++r) {
                    u0[r] = T(0);
                    u1[r] = T(0);
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        g0[a][r] = T(0);
                        g1[a][r] = T(0);
                    }
                }
                {
                    const T* u = sU + te * BS;
                    const T* Eq = op.E_q + f * NBF * nq + q;
                    const T* Dq = op.Dxi_q + f * NBF * D * nq + q;
                    for (int k = 0; k < NBF; ++k) {
                        const T ev = __ldg(&Eq[k * nq]);
#pragma unroll
                        for (int r = 0; r < Q; ++r) u0[r] += ev * u[k + NBF * r];
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            const T dv = __ldg(&Dq[(k * D + a) * nq]);
#pragma unroll
                            for (int r = 0; r < Q; ++r) g0[a][r] += dv * u[k + NBF * r];
                        }
                    }
                }
                if (mode == 1) {
                    const T* u = sUn + te * BS;
                    const T* Eq = op.E_q + nbl * NBF * nq + q;
                    const T* Dq = op.Dxi_q + nbl * NBF * D * nq + q;
                    for (int k = 0; k < NBF; ++k) {
                        const T ev = __ldg(&Eq[k * nq]);
#pragma unroll
                        for (int r = 0; r < Q; ++r) u1[r] += ev * u[k + NBF * r];
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            const T dv = __ldg(&Dq[(k * D + a) * nq]);
#pragma unroll
                            for (int r = 0; r < Q; ++r) g1[a][r] += dv * u[k + NBF * r];
                        }
                    }
                }
                T n[D], nu[D];
#pragma unroll
                for (int i = 0; i < D; ++i) {
                    n[i] = flip * op.fN[(static_cast<int64_t>(fct) * D + i) * nq + q];
                    nu[i] = flip * op.fNunit[(static_cast<int64_t>(fct) * D + i) * nq + q];
                }
                const double pen = op.penalty[fct];
                const T wq = op.w[q];

                if constexpr (S::KIND == kPoisson) {
                    T KG0[DD], KG1[DD];
                    const T* kg = op.fCoef + static_cast<int64_t>(fct) * 2 * DD * nq + q;
#pragma unroll
                    for (int c = 0; c < DD; ++c) {
                        KG0[c] = kg[(own * DD + c) * nq];
                        KG1[c] = kg[(oth * DD + c) * nq];
                    }
                    T uh, sig[D];
                    if (mode == 1) {
                        uh = T(0.5) * (u1[0] - u0[0]);
                        const T pj = static_cast<T>(pen * static_cast<double>(u0[0] - u1[0]));
#pragma unroll
                        for (int p = 0; p < D; ++p) {
                            T s = T(0);
#pragma unroll
                            for (int a = 0; a < D; ++a) s += KG0[a * D + p] * g0[a][0] + KG1[a * D + p] * g1[a][0];
                            sig[p] = T(0.5) * s - pj * nu[p];
                        }
                    } else {
                        uh = -u0[0];
                        const T pj = static_cast<T>(pen * static_cast<double>(u0[0]));
#pragma unroll
                        for (int p = 0; p < D; ++p) {
                            T s = T(0);
#pragma unroll
                            for (int a = 0; a < D; ++a) s += KG0[a * D + p] * g0[a][0];
                            sig[p] = s - pj * nu[p];
                        }
                    }
                    T bsum = T(0);
#pragma unroll
                    for (int r = 0; r < D; ++r) bsum += n[r] * sig[r];
                    b_out[0] = -wq * bsum;
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        T s = T(0);
#pragma unroll
                        for (int r = 0; r < D; ++r) s += n[r] * KG0[a * D + r];
                        a_out[a * nq] = wq * uh * s;
                    }
                } else {
                    T G0[DD], G1[DD];
                    const T* gg = op.fG + static_cast<int64_t>(fct) * 2 * DD * nq + q;
#pragma unroll
                    for (int c = 0; c < DD; ++c) {
                        G0[c] = gg[(own * DD + c) * nq];
                        G1[c] = gg[(oth * DD + c) * nq];
                    }
                    const T* lm = op.fCoef + static_cast<int64_t>(fct) * 4 * nq + q;
                    const T lam0 = lm[(2 * own + 0) * nq], mu0 = lm[(2 * own + 1) * nq];
                    const T lam1 = lm[(2 * oth + 0) * nq], mu1 = lm[(2 * oth + 1) * nq];
                    // Ju[s][r] = d u_r / d x_s on each side
                    T sg[D][D];
                    {
                        T J0[D][D];
#pragma unroll
                        for (int s = 0; s < D; ++s)
#pragma unroll
                            for (int r = 0; r < D; ++r) {
                                T acc0 = T(0);
#pragma unroll
                                for (int a = 0; a < D; ++a) acc0 += G0[a * D + s] * g0[a][r];
                                J0[s][r] = acc0;
                            }
                        T d0 = T(0);
#pragma unroll
                        for (int r = 0; r < D; ++r) d0 += J0[r][r];
#pragma unroll
                        for (int i = 0; i < D; ++i)
#pragma unroll
                            for (int j = 0; j < D; ++j)
                                sg[i][j] = mu0 * (J0[i][j] + J0[j][i]) + ((i == j) ? lam0 * d0 : T(0));
                    }
                    T uhm[D];
                    if (mode == 1) {
                        T J1[D][D];
#pragma unroll
                        for (int s = 0; s < D; ++s)
#pragma unroll
                            for (int r = 0; r < D; ++r) {
                                T acc1 = T(0);
#pragma unroll
                                for (int a = 0; a < D; ++a) acc1 += G1[a * D + s] * g1[a][r];
                                J1[s][r] = acc1;
                            }
                        T d1 = T(0);
#pragma unroll
                        for (int r = 0; r < D; ++r) d1 += J1[r][r];
#pragma unroll
                        for (int i = 0; i < D; ++i) {
                            const T pj = static_cast<T>(pen * static_cast<double>(u0[i] - u1[i]));
#pragma unroll
                            for (int j = 0; j < D; ++j) {
                                const T s1 = mu1 * (J1[i][j] + J1[j][i]) + ((i == j) ? lam1 * d1 : T(0));
                                sg[i][j] = T(0.5) * (sg[i][j] + s1) - pj * nu[j];
                            }
                            uhm[i] = T(0.5) * (u1[i] - u0[i]);
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < D; ++i) {
                            const T pj = static_cast<T>(pen * static_cast<double>(u0[i]));
#pragma unroll
                            for (int j = 0; j < D; ++j) sg[i][j] = sg[i][j] - pj * nu[j];
                            uhm[i] = -u0[i];
                        }
                    }
                    T un = T(0);
#pragma unroll
                    for (int r = 0; r < D; ++r) un += uhm[r] * n[r];
#pragma unroll
                    for (int uu = 0; uu < D; ++uu) {
                        T X[D];
#pragma unroll
                        for (int j = 0; j < D; ++j)
                            X[j] = mu0 * (uhm[uu] * n[j] + uhm[j] * n[uu]) + ((uu == j) ? lam0 * un : T(0));
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            T s = T(0);
#pragma unroll
                            for (int j = 0; j < D; ++j) s += G0[a * D + j] * X[j];
                            a_out[(uu * D + a) * nq] = wq * s;
                        }
                        T bsum = T(0);
#pragma unroll
                        for (int j = 0; j < D; ++j) bsum += n[j] * sg[uu][j];
                        b_out[uu * nq] = -wq * bsum;
                    }
                }
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                const int it = tid + j * NT;
                if (it < TE * BS) {
                    const int te = it / BS, rem = it - te * BS;
                    const int uu = rem / NBF, k = rem - uu * NBF;
                    const T* a = sA + (te * Q + uu) * D * nq;
                    const T* b = sB + (te * Q + uu) * nq;
                    const T* DT = op.DxiT_q + f * D * nq * NBF + k;
                    const T* ET = op.ET_q + f * nq * NBF + k;
                    T s = T(0);
                    for (int c = 0; c < D * nq; ++c) s += __ldg(&DT[c * NBF]) * a[c];
                    for (int q = 0; q < nq; ++q) s += __ldg(&ET[q * NBF]) * b[q];
                    acc[j] += s;
                }
            }
        }

#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const int it = tid + j * NT;
            if (it < TE * BS && e0 + it / BS < E) y[e0 * BS + it] = acc[j];
        }
    }
}

}  // namespace tdg
