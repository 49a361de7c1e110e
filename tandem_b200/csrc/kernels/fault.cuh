// Fault coupling of the Poisson operator, batched over right-hand sides (Green's functions).
//
//  slip -> rhs:   slip coefficients on each fault facet (nodal fault basis of degree N) evaluated
//                 at the facet points with tandem's sign convention (Adapter<Poisson>::slip,
//                 app/localoperator/PoissonAdapter.cpp:36-55), then the interior-penalty
//                 skeleton / boundary load (Poisson::rhs_skeleton / rhs_boundary with the IP lift,
//                 Poisson.cpp:434-549; a fault facet on the boundary carries half the slip,
//                 Poisson.cpp:418-432).
//  u -> traction: grad_u on the fault (poisson.py:146-152, Poisson::traction_skeleton /
//                 traction_boundary, Poisson.cpp:678-723) projected on the fault basis with the
//                 fault mass matrix (evaluate_traction, poisson_adapter.py:21-23,
//                 PoissonAdapter.cpp:22-34).
// One CTA per (fault facet, right-hand side); a CTA whose slip vanishes on its facet returns at
// once, so the Green's-function batch (one unit slip per right-hand side) costs two facets' work
// per column.
#pragma once

#include "common.cuh"

namespace tdg {

struct DevFault {
    int nfault = 0, nbf = 0;         // fault facets, fault basis functions per facet
    const int4* info = nullptr;      // [nfault] {facet, up0, up1, loc0 | loc1 << 8}
    const double* sign = nullptr;    // [nfault][nq] +1 / -1 (fault normal vs side-0 facet normal)
    const double* normal = nullptr;  // [nfault][D][nq] fault normal (|detJ|-scaled, oriented)
    const double* minv = nullptr;    // [nfault][nbf][nbf] inverse fault mass matrix
    const double* e_q = nullptr;     // [nbf][nq] fault basis at the facet points
};

constexpr int kFaultThreads = 128;
constexpr int kFaultMaxQ = 64;

// slip [rhs][nfault][nbf] (leading dimension ld_slip) -> b += rhs contributions.
template <class S>
__global__ void __launch_bounds__(kFaultThreads)
    fault_rhs_kernel(DevOp<double> op, DevFault fl, const double* __restrict__ slip, int64_t ld_slip,
                     double* __restrict__ b, int64_t ld) {
    constexpr int D = S::D, NBF = S::NBF, DD = S::DD;
    const int nq = op.nq;
    const int fi = blockIdx.x, rhs = blockIdx.y, tid = threadIdx.x;
    __shared__ double fq[kFaultMaxQ];
    __shared__ int any;
    if (tid == 0) any = 0;
    __syncthreads();
    const double* sl = slip + rhs * ld_slip + static_cast<int64_t>(fi) * fl.nbf;
    const int4 info = fl.info[fi];
    const int fct = info.x;
    const bool boundary = info.y == info.z;
    for (int q = tid; q < nq; q += blockDim.x) {
        double s = 0.0;
        for (int p = 0; p < fl.nbf; ++p) s += fl.e_q[p * nq + q] * sl[p];
        s *= fl.sign[static_cast<int64_t>(fi) * nq + q];
        if (boundary) s *= 0.5;
        fq[q] = s;
        if (s != 0.0) any = 1;
    }
    __syncthreads();
    if (!any) return;
    const double pen = op.penalty[fct];
    for (int side = 0; side < (boundary ? 1 : 2); ++side) {
        const int el = side == 0 ? info.y : info.z;
        const int l = side == 0 ? (info.w & 0xff) : (info.w >> 8);
        const double c10 = boundary ? -1.0 : -0.5;
        const double c20 = side == 0 ? pen : -pen;
        for (int k = tid; k < NBF; k += blockDim.x) {
            double s1 = 0.0, s2 = 0.0;
            for (int q = 0; q < nq; ++q) {
                const double wq = op.w[q];
                double dn = 0.0;
                for (int i = 0; i < D; ++i) {
                    double kd = 0.0;
#pragma unroll
                    for (int e = 0; e < D; ++e)
                        kd += op.fCoef[((static_cast<int64_t>(fct) * 2 + side) * DD + e * D + i) * nq + q] *
                              op.Dxi_q[((l * NBF + k) * D + e) * nq + q];
                    dn += kd * op.fN[(static_cast<int64_t>(fct) * D + i) * nq + q];
                }
                s1 += wq * dn * fq[q];
                s2 += wq * op.E_q[(l * NBF + k) * nq + q] * op.fNl[static_cast<int64_t>(fct) * nq + q] * fq[q];
            }
            atomicAdd(&b[rhs * ld + static_cast<int64_t>(el) * NBF + k], c10 * s1 + c20 * s2);
        }
    }
}

// u [rhs][ld], slip [rhs][ld_slip] -> traction [rhs][nfault][nbf] (leading dimension ld_t).
template <class S>
__global__ void __launch_bounds__(kFaultThreads)
    fault_traction_kernel(DevOp<double> op, DevFault fl, const double* __restrict__ u, int64_t ld,
                          const double* __restrict__ slip, int64_t ld_slip, double* __restrict__ traction,
                          int64_t ld_t) {
    constexpr int D = S::D, NBF = S::NBF, DD = S::DD;
    const int nq = op.nq;
    const int fi = blockIdx.x, rhs = blockIdx.y, tid = threadIdx.x;
    __shared__ double sq[kFaultMaxQ];
    const int4 info = fl.info[fi];
    const int fct = info.x;
    const bool boundary = info.y == info.z;
    const int l0 = info.w & 0xff, l1 = info.w >> 8;
    const double* u0 = u + rhs * ld + static_cast<int64_t>(info.y) * NBF;
    const double* u1 = u + rhs * ld + static_cast<int64_t>(info.z) * NBF;
    const double* sl = slip ? slip + rhs * ld_slip + static_cast<int64_t>(fi) * fl.nbf : nullptr;
    const double pen = op.penalty[fct];
    for (int q = tid; q < nq; q += blockDim.x) {
        double f = 0.0;
        if (sl) {
            for (int p = 0; p < fl.nbf; ++p) f += fl.e_q[p * nq + q] * sl[p];
            f *= fl.sign[static_cast<int64_t>(fi) * nq + q];
            if (boundary) f *= 0.5;
        }
        double g0[D], g1[D], e0 = 0.0, e1 = 0.0;
#pragma unroll
        for (int e = 0; e < D; ++e) g0[e] = g1[e] = 0.0;
        for (int k = 0; k < NBF; ++k) {
            e0 += op.E_q[(l0 * NBF + k) * nq + q] * u0[k];
#pragma unroll
            for (int e = 0; e < D; ++e) g0[e] += op.Dxi_q[((l0 * NBF + k) * D + e) * nq + q] * u0[k];
            if (!boundary) {
                e1 += op.E_q[(l1 * NBF + k) * nq + q] * u1[k];
#pragma unroll
                for (int e = 0; e < D; ++e) g1[e] += op.Dxi_q[((l1 * NBF + k) * D + e) * nq + q] * u1[k];
            }
        }
        double s = 0.0;
#pragma unroll
        for (int p = 0; p < D; ++p) {
            double k0 = 0.0, k1 = 0.0;
#pragma unroll
            for (int e = 0; e < D; ++e) {
                k0 += op.fCoef[((static_cast<int64_t>(fct) * 2 + 0) * DD + e * D + p) * nq + q] * g0[e];
                k1 += op.fCoef[((static_cast<int64_t>(fct) * 2 + 1) * DD + e * D + p) * nq + q] * g1[e];
            }
            const double nu = op.fNunit[(static_cast<int64_t>(fct) * D + p) * nq + q];
            const double grad = boundary ? (k0 - pen * (e0 - f) * nu) : (0.5 * (k0 + k1) - pen * (e0 - e1 - f) * nu);
            s += grad * fl.normal[(static_cast<int64_t>(fi) * D + p) * nq + q];
        }
        sq[q] = op.w[q] * s;
    }
    __syncthreads();
    for (int p = tid; p < fl.nbf; p += blockDim.x) {
        double t = 0.0;
        for (int r = 0; r < fl.nbf; ++r) {
            double a = 0.0;
            for (int q = 0; q < nq; ++q) a += fl.e_q[r * nq + q] * sq[q];
            t += fl.minv[(static_cast<int64_t>(fi) * fl.nbf + r) * fl.nbf + p] * a;
        }
        traction[rhs * ld_t + static_cast<int64_t>(fi) * fl.nbf + p] = t;
    }
}

}  // namespace tdg
