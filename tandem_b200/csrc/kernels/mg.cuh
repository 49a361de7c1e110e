// p-multigrid preconditioner kernels (tandem's PCMG configuration, app/common/PetscLinearSolver.cpp:53-114
// with examples/options/mg_cheby.cfg: Chebyshev + point-Jacobi smoothing on every level, Galerkin
// coarse operators A_l = I^T A_{l+1} I, a Krylov coarse solve).
//
// Level matrices are element block-sparse: block row e holds NB = 1 + nfaces blocks of bs x bs
// doubles, column-major (blk[col * bs + row], row = k + Nbf p), slot 0 the element itself and
// slot 1 + f the element behind local face f (nbr[e][s] < 0: no block; a boundary facet's
// coupling is part of the self block).  The interpolation is block diagonal over elements and
// components with one reference matrix I [N1][N2] (fine basis k, coarse basis l).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tdg {

struct MgInterp {
    const double* I;  // [N1][N2] row-major, device
    int N1, N2, Q;    // fine and coarse basis sizes, components
};

// Probing of the matrix-free operator: V (nj columns of leading dimension ld, zeroed by the
// caller) gets, on every element of colour c, column j0 + jj of the element interpolation.
int launch_mg_probe_fill(int64_t E, const int32_t* colour, int c, MgInterp ip, int j0, int nj, double* V,
                         int64_t ld, cudaStream_t s);
// A[n][s][:, j0 + jj] = I^T Y_n[:, jj] for every block (n, s) whose element nbr[n][s] has colour c
// (each closed neighbourhood holds a colour at most once, so Y_n is that block's column alone).
int launch_mg_probe_extract(int64_t E, int NB, const int32_t* nbr, const int32_t* colour, int c, MgInterp ip,
                            int j0, int nj, const double* Y, int64_t ld, double* A, cudaStream_t s);
// Ac[n][s] = I^T Af[n][s] I for every present block.
int launch_mg_triple(int64_t E, int NB, const int32_t* nbr, MgInterp ip, const double* Af, double* Ac,
                     cudaStream_t s);
// y = A x (b == nullptr) or y = b - A x, for nrhs columns starting at multiples of ld.
template <typename TA>
int launch_mg_bsr_apply(int64_t E, int NB, int bs, const int32_t* nbr, const TA* A, const double* x,
                        const double* b, double* y, int nrhs, int64_t ld, cudaStream_t s);
// b[i] = a[i] rounded to FP32 (the mixed-precision smoother's copies of the level blocks).
int launch_round_to_float(int64_t n, const double* a, float* b, cudaStream_t s);
// dinv[e][i] = 1 / blocks[e * stride + i * bs + i] (point Jacobi); status set on a non-positive
// diagonal entry.
int launch_mg_diag_inv(int64_t E, int bs, int64_t stride, const double* blocks, double* dinv, int* status,
                       cudaStream_t s);
// blk[e] = A[e][0] (self blocks, contiguous, for the block-Jacobi inversion).
int launch_mg_self_blocks(int64_t E, int NB, int bs, const double* A, double* blk, cudaStream_t s);
// xf += I xc; rc = I^T rf (nrhs columns, leading dimensions ldc / ldf).
int launch_mg_prolong_add(int64_t E, MgInterp ip, const double* xc, int64_t ldc, double* xf, int64_t ldf, int nrhs,
                          cudaStream_t s);
int launch_mg_restrict(int64_t E, MgInterp ip, const double* rf, int64_t ldf, double* rc, int64_t ldc, int nrhs,
                       cudaStream_t s);

// Continuous P1 auxiliary level: R maps vertex values to the coarsest DG level (on element e, corner
// values through T [Nbf][NV] per component); its Galerkin operator is CSR over vertices with Q x Q
// blocks (row-major).  The restriction gathers over each vertex's (element, corner) incidences, so
// it needs no atomics and is deterministic.
struct MgAux {
    const int64_t* ptr = nullptr;
    const int32_t* col = nullptr;
    const double* val = nullptr;
    const int64_t* vinc_ptr = nullptr;
    const int32_t* vinc = nullptr;  // e * NV + corner
    const int32_t* vid = nullptr;   // [E][NV]
    const double* T = nullptr;      // [Nbf][NV]
    int64_t nv = 0;
    int Q = 0, Nbf = 0, NV = 0;
};
// P1 vectors: nrhs contiguous columns of nv * Q; DG level columns at multiples of ld0.
int launch_aux_apply(MgAux const& a, const double* x, const double* b, double* y, int nrhs, cudaStream_t s);
int launch_aux_restrict(MgAux const& a, const double* r0, int64_t ld0, double* rc, int nrhs, cudaStream_t s);
int launch_aux_prolong_add(MgAux const& a, int64_t E, const double* xc, double* x0, int64_t ld0, int nrhs,
                           cudaStream_t s);

// Chebyshev iteration (Saad, "Iterative Methods for Sparse Linear Systems", 2nd ed., Alg. 12.1,
// preconditioned with Dinv): first step d = c Dinv r, x = d (x_zero) or x += d; later steps
// r -= y (y = A d), d = c1 d + c2 Dinv r, x += d.  nrhs columns of n entries at stride ld.
int launch_cheb_first(int64_t n, int nrhs, int64_t ld, const double* dinv, const double* r, double* d, double* x,
                      double c, int x_zero, cudaStream_t s);
int launch_cheb_step(int64_t n, int nrhs, int64_t ld, const double* dinv, const double* y, double* r, double* d,
                     double* x, double c1, double c2, cudaStream_t s);
// y = x and y = a - y over nrhs columns of n entries at stride ld (padding untouched).
int launch_vec_copy_cols(int64_t n, int nrhs, int64_t ld, const double* x, double* y, cudaStream_t s);
int launch_vec_rsub_cols(int64_t n, int nrhs, int64_t ld, const double* a, double* y, cudaStream_t s);

// Vector helpers of the level solvers (grid-stride).  dot: deterministic two-pass sum into
// out[0] (partial holds kDotBlocks doubles).
constexpr int kDotBlocks = 592;
int launch_vec_dot(int64_t n, const double* a, const double* b, double* partial, double* out, cudaStream_t s);
int launch_vec_axpby(int64_t n, double a, const double* x, double b, double* y, cudaStream_t s);  // y = a x + b y
int launch_vec_mul(int64_t n, const double* a, const double* x, double* y, cudaStream_t s);        // y = a .* x
int launch_vec_sub(int64_t n, const double* a, const double* b, double* y, cudaStream_t s);        // y = a - b (y may be b)
int launch_vec_random(int64_t n, uint64_t seed, double* y, cudaStream_t s);                        // uniform [-1, 1)

}  // namespace tdg
