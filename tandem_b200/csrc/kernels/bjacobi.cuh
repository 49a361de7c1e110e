// Block-Jacobi preconditioner on the device.
//
// assemble: the element diagonal block D_e = A_vol(e) + sum over the element's faces of the
//   facet self block (tandem's DGOperator::assemble restricted to A(e, e),
//   src/form/DGOperator.h:121-187, with Poisson::assemble_volume/skeleton/boundary,
//   app/localoperator/Poisson.cpp:225-385, and Elasticity::assemble_*, Elasticity.cpp:317-519;
//   IP lift, interior constants c00 = c10 = -1/2, boundary -1, c20 = penalty).  Blocks are
//   column-major: blk[e][col * BS + row], row = k + NBF p.
// invert: Gauss-Jordan without pivoting in shared memory; a non-positive pivot marks the block
//   as not positive definite (SIPG diagonal blocks are SPD for a sufficient penalty).
// apply: z_e = D_e^-1 r_e, one thread per (element, row), inverse streamed column by column.
#pragma once

#include "common.cuh"

namespace tdg {

template <class S>
__host__ __device__ inline int bjac_assemble_smem_doubles(int Nq, int nq) {
    int vol = S::NBF * S::D * Nq + 2 * Nq;
    int fct = S::NBF * S::D * nq + S::NBF * nq + (S::D + 2 + 2) * nq;
    return vol > fct ? vol : fct;
}

template <class S>
__global__ void __launch_bounds__(256) bjac_assemble_kernel(DevOp<double> op, double* __restrict__ blk) {
    constexpr int D = S::D, NBF = S::NBF, Q = S::Q, BS = S::BS, DD = S::DD, NF = S::NF;
    const int Nq = op.Nq, nq = op.nq;
    const int64_t e = blockIdx.x;
    const int tid = threadIdx.x;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sm = reinterpret_cast<double*>(smem_raw);
    double* out = blk + e * BS * BS;

    // volume: physical gradients Dx[k][i][q]
    double* sDx = sm;
    double* sC = sm + NBF * D * Nq;
    for (int it = tid; it < NBF * D * Nq; it += blockDim.x) {
        const int q = it % Nq;
        const int i = (it / Nq) % D;
        const int k = it / (Nq * D);
        double s = 0.0;
        for (int a = 0; a < D; ++a)
            s += op.vG[(e * DD + a * D + i) * Nq + q] * op.Dxi_Q[(k * D + a) * Nq + q];
        sDx[it] = s;
    }
    const int ncoef = (S::KIND == kPoisson) ? 1 : 2;
    for (int it = tid; it < ncoef * Nq; it += blockDim.x) sC[it] = op.vCoef[e * ncoef * Nq + it];
    __syncthreads();
    for (int it = tid; it < BS * BS; it += blockDim.x) {
        const int row = it % BS, col = it / BS;
        const int k = row % NBF, p = row / NBF, l = col % NBF, u = col / NBF;
        double s = 0.0;
        if constexpr (S::KIND == kPoisson) {
            for (int q = 0; q < Nq; ++q) {
                double d = 0.0;
                for (int i = 0; i < D; ++i) d += sDx[(k * D + i) * Nq + q] * sDx[(l * D + i) * Nq + q];
                s += sC[q] * d;
            }
        } else {
            for (int q = 0; q < Nq; ++q) {
                const double lam = sC[q], mu = sC[Nq + q];
                double kl = 0.0;
                for (int j = 0; j < D; ++j) kl += sDx[(k * D + j) * Nq + q] * sDx[(l * D + j) * Nq + q];
                s += lam * sDx[(k * D + p) * Nq + q] * sDx[(l * D + u) * Nq + q] +
                     mu * ((p == u ? kl : 0.0) + sDx[(k * D + u) * Nq + q] * sDx[(l * D + p) * Nq + q]);
            }
        }
        out[it] = s;
    }

    // facet self blocks
    for (int f = 0; f < NF; ++f) {
        const int4 sd = op.sides[e * NF + f];
        const int bcv = sd.y >> 8;
        const bool skel = sd.z != static_cast<int>(e);
        if (!skel && !(bcv == 3 || bcv == 5)) continue;
        const int fct = sd.x;
        const int own = skel ? (sd.y & 0xff) : 0;
        const double flip = (skel && own == 1) ? -1.0 : 1.0;
        const double c = skel ? -0.5 : -1.0;
        const double pen = op.penalty[fct];
        __syncthreads();
        double* fDx = sm;                       // [NBF][D][nq]  (Poisson: K * Dx)
        double* fE = fDx + NBF * D * nq;        // [NBF][nq]
        double* fn = fE + NBF * nq;             // [D][nq] outward normal
        double* fnl = fn + D * nq;              // [nq]
        double* fc = fnl + nq;                  // [2][nq] lam, mu
        for (int it = tid; it < NBF * D * nq; it += blockDim.x) {
            const int q = it % nq;
            const int i = (it / nq) % D;
            const int k = it / (nq * D);
            double s = 0.0;
            for (int a = 0; a < D; ++a) {
                double g;
                if constexpr (S::KIND == kPoisson) {
                    g = op.fCoef[((static_cast<int64_t>(fct) * 2 + own) * DD + a * D + i) * nq + q];
                } else {
                    g = op.fG[((static_cast<int64_t>(fct) * 2 + own) * DD + a * D + i) * nq + q];
                }
                s += g * op.Dxi_q[((f * NBF + k) * D + a) * nq + q];
            }
            fDx[it] = s;
        }
        for (int it = tid; it < NBF * nq; it += blockDim.x) fE[it] = op.E_q[f * NBF * nq + it];
        for (int it = tid; it < D * nq; it += blockDim.x)
            fn[it] = flip * op.fN[static_cast<int64_t>(fct) * D * nq + it];
        for (int it = tid; it < nq; it += blockDim.x) {
            fnl[it] = op.fNl[static_cast<int64_t>(fct) * nq + it];
            if constexpr (S::KIND != kPoisson) {
                fc[it] = op.fCoef[(static_cast<int64_t>(fct) * 4 + 2 * own + 0) * nq + it];
                fc[nq + it] = op.fCoef[(static_cast<int64_t>(fct) * 4 + 2 * own + 1) * nq + it];
            }
        }
        __syncthreads();
        for (int it = tid; it < BS * BS; it += blockDim.x) {
            const int row = it % BS, col = it / BS;
            const int k = row % NBF, p = row / NBF, l = col % NBF, u = col / NBF;
            double s = 0.0;
            for (int q = 0; q < nq; ++q) {
                const double wq = op.w[q];
                const double ek = fE[k * nq + q], el = fE[l * nq + q];
                if constexpr (S::KIND == kPoisson) {
                    double dk = 0.0, dl = 0.0;
                    for (int i = 0; i < D; ++i) {
                        dk += fDx[(k * D + i) * nq + q] * fn[i * nq + q];
                        dl += fDx[(l * D + i) * nq + q] * fn[i * nq + q];
                    }
                    s += wq * (c * dk * el + c * dl * ek + pen * ek * el * fnl[q]);
                } else {
                    const double lam = fc[q], mu = fc[nq + q];
                    double dkn = 0.0, dln = 0.0;
                    for (int j = 0; j < D; ++j) {
                        dkn += fDx[(k * D + j) * nq + q] * fn[j * nq + q];
                        dln += fDx[(l * D + j) * nq + q] * fn[j * nq + q];
                    }
                    // traction operator T[m, a, b] = lam Dx[m,a] n_b + mu (dmn delta_ab + Dx[m,b] n_a)
                    const double Tl = lam * fDx[(l * D + u) * nq + q] * fn[p * nq + q] +
                                      mu * ((u == p ? dln : 0.0) + fDx[(l * D + p) * nq + q] * fn[u * nq + q]);
                    const double Tk = lam * fDx[(k * D + p) * nq + q] * fn[u * nq + q] +
                                      mu * ((p == u ? dkn : 0.0) + fDx[(k * D + u) * nq + q] * fn[p * nq + q]);
                    s += wq * (c * ek * Tl + c * el * Tk + (p == u ? pen * ek * el * fnl[q] : 0.0));
                }
            }
            out[it] += s;
        }
    }
}

// In-place Gauss-Jordan inversion of one BS x BS block per CTA; writes the inverse in T.
template <int BS, typename T>
__global__ void __launch_bounds__(256)
    bjac_invert_kernel(const double* __restrict__ blk, T* __restrict__ inv, int* __restrict__ status) {
    const int64_t e = blockIdx.x;
    const int tid = threadIdx.x;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* a = reinterpret_cast<double*>(smem_raw);  // column-major a[col * BS + row]
    double* colk = a + BS * BS;                       // copy of column k
    __shared__ int bad;
    if (tid == 0) bad = 0;
    for (int i = tid; i < BS * BS; i += blockDim.x) a[i] = blk[e * BS * BS + i];
    __syncthreads();
    for (int k = 0; k < BS; ++k) {
        double piv = a[k * BS + k];
        if (!(piv > 0.0)) {
            if (tid == 0) bad = 1;
            piv = 1.0;
        }
        const double ip = 1.0 / piv;
        // save column k (multipliers), then scale row k
        for (int i = tid; i < BS; i += blockDim.x) colk[i] = a[k * BS + i];
        __syncthreads();
        for (int j = tid; j < BS; j += blockDim.x) a[j * BS + k] = (j == k ? 1.0 : a[j * BS + k]) * ip;
        __syncthreads();
        for (int it = tid; it < BS * BS; it += blockDim.x) {
            const int i = it % BS, j = it / BS;
            if (i == k) continue;
            const double fi = colk[i];
            const double rk = a[j * BS + k];
            a[it] = (j == k ? 0.0 : a[it]) - fi * rk;
        }
        __syncthreads();
    }
    for (int i = tid; i < BS * BS; i += blockDim.x) inv[e * BS * BS + i] = static_cast<T>(a[i]);
    if (tid == 0 && bad) atomicOr(status, 1);
}

// z = Dinv r for nrhs vectors: one thread per (element, row).
template <int BS, typename TM, typename TV>
__global__ void __launch_bounds__(256) bjac_apply_kernel(int64_t E, const TM* __restrict__ inv,
                                                         const TV* __restrict__ r, TV* __restrict__ z,
                                                         int64_t ld) {
    constexpr int TE = (256 / BS) > 0 ? (256 / BS) : 1;
    __shared__ TV sr[TE * BS];
    const int rhs = blockIdx.y;
    r += rhs * ld;
    z += rhs * ld;
    const int64_t ntiles = (E + TE - 1) / TE;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t e0 = tile * TE;
        __syncthreads();
        for (int i = threadIdx.x; i < TE * BS; i += blockDim.x)
            sr[i] = (e0 + i / BS < E) ? r[e0 * BS + i] : TV(0);
        __syncthreads();
        const int te = threadIdx.x / BS, row = threadIdx.x % BS;
        const int64_t e = e0 + te;
        if (te < TE && e < E) {
            const TM* m = inv + e * BS * BS + row;
            const TV* rv = sr + te * BS;
            TV s = TV(0);
#pragma unroll 8
            for (int c = 0; c < BS; ++c) s += static_cast<TV>(m[c * BS]) * rv[c];
            z[e * BS + row] = s;
        }
    }
}

}  // namespace tdg
