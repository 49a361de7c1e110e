// Explicit wave operator of elasticity (tandem's Elasticity::wave_rhs,
// app/localoperator/Elasticity.cpp:865-880): the right-hand side of rho u'' = -A u + b is
// M^-1 (b - A u) / rho, evaluated as tandem's apply_inverse_mass kernel
// (app/kernels/elasticity.py:236-237):
//
//   Unew(k, p) = Minv(k, r) E_Q(r, q) nrwj(q) E_Q(s, q) Minv(s, l) U(l, p),
//   nrwj(q) = -rhoInv(x_q) W_q / |J|_q,
//
// with Minv the reference element's inverse mass matrix (exact element inverse mass for affine
// elements, tandem's approximation on curved ones).  One CTA per element; in place is allowed
// (the block is read into shared memory before it is written).
#pragma once

#include "common.cuh"

namespace tdg {

struct WaveData {
    const double* EQ = nullptr;    // [NBF][Nq] basis values at the volume points
    const double* Minv = nullptr;  // [NBF][NBF] reference inverse mass (row-major)
    const double* nrwj = nullptr;  // [E][Nq]
};

constexpr int kWaveThreads = 128;

template <class S>
__global__ void __launch_bounds__(kWaveThreads)
    inverse_mass_kernel(WaveData wd, int64_t E, int Nq, const double* x, const double* b, double* y, int64_t ld) {
    constexpr int NBF = S::NBF, Q = S::Q, BS = S::BS;
    const int64_t e = blockIdx.x;
    const int rhs = blockIdx.y;
    x += rhs * ld;
    y += rhs * ld;
    if (b) b += rhs * ld;
    extern __shared__ double sh[];
    double* U = sh;               // [BS]   (x - b) block
    double* A = U + BS;           // [BS]   Minv U
    double* Wq = A + BS;          // [Nq][Q]
    const int tid = threadIdx.x;
    for (int i = tid; i < BS; i += blockDim.x)
        U[i] = x[e * BS + i] - (b ? b[e * BS + i] : 0.0);
    __syncthreads();
    for (int i = tid; i < BS; i += blockDim.x) {
        const int k = i % NBF, p = i / NBF;
        double s = 0.0;
        for (int l = 0; l < NBF; ++l) s += wd.Minv[k * NBF + l] * U[l + NBF * p];
        A[i] = s;
    }
    __syncthreads();
    for (int i = tid; i < Nq * Q; i += blockDim.x) {
        const int q = i % Nq, p = i / Nq;
        double s = 0.0;
        for (int k = 0; k < NBF; ++k) s += wd.EQ[k * Nq + q] * A[k + NBF * p];
        Wq[q + Nq * p] = s * wd.nrwj[e * Nq + q];
    }
    __syncthreads();
    for (int i = tid; i < BS; i += blockDim.x) {  // A <- E_Q Wq
        const int r = i % NBF, p = i / NBF;
        double s = 0.0;
        for (int q = 0; q < Nq; ++q) s += wd.EQ[r * Nq + q] * Wq[q + Nq * p];
        U[i] = s;
    }
    __syncthreads();
    for (int i = tid; i < BS; i += blockDim.x) {
        const int k = i % NBF, p = i / NBF;
        double s = 0.0;
        for (int r = 0; r < NBF; ++r) s += wd.Minv[k * NBF + r] * U[r + NBF * p];
        y[e * BS + i] = s;
    }
}

}  // namespace tdg
