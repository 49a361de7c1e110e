/*
 * tandem_b200 C ABI: the device (sm_100a) matrix-free DG operator behind tandem's MatShell.
 *
 * Every entry point is plain C: pointers, sizes and an opaque handle.  Device arrays are CUDA
 * device pointers; `stream` is a cudaStream_t passed as void* (NULL = the legacy default stream).
 * All device work is enqueued on `stream` and returns without synchronising unless stated.
 * Return value: 0 on success, a negative TDG_E* code otherwise; tdg_last_error() gives the text.
 * No exception crosses this boundary.
 *
 * Vector layout (tandem's BlockVector over a PETSc Vec, app/common/PetscVector.h:48-56):
 * one block of bs = Nbf * Q values per element, basis index fastest, then component:
 * x[e * bs + k + Nbf * p].  Multi-RHS vectors stack nrhs such vectors with leading dimension ld
 * (ld >= E * bs): x[r * ld + e * bs + k + Nbf * p].
 */
#ifndef TANDEM_B200_H
#define TANDEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes. */
#define TDG_OK 0
#define TDG_E_INVALID (-1)     /* invalid argument */
#define TDG_E_CUDA (-2)        /* CUDA runtime error */
#define TDG_E_NOT_SPD (-3)     /* a block-Jacobi diagonal block is not positive definite */
#define TDG_E_DIVERGED (-4)    /* Krylov solve did not converge / produced NaN */
#define TDG_E_STATE (-5)       /* call out of order (e.g. apply before set_material) */
#define TDG_E_TIMEOUT (-6)     /* a bounded device wait ran out */
#define TDG_E_NOMEM (-7)       /* device allocation failed */

/* Local operator kind: tandem's Poisson (app/localoperator/Poisson.h:31) and
 * Elasticity (app/localoperator/Elasticity.h:31). */
#define TDG_POISSON 0
#define TDG_ELASTICITY 1

/* Facet boundary conditions, values of tandem's enum class BC (src/form/BC.h:6). */
#define TDG_BC_NONE 0
#define TDG_BC_NATURAL 1
#define TDG_BC_FAULT 3
#define TDG_BC_DIRICHLET 5

/* Arithmetic of an apply / preconditioner / solve.  TDG_MIXED: FP32 operator arithmetic (and FP32
 * block inverses) on FP64 vectors; as a solve precision, an FP64 CG recurrence around them.
 * TDG_TF32: FP64 vectors, the operator's products in one TF32 tensor-core pass (about 1e-3 of
 * |A| |x|; TDG_MIXED runs three, 3xTF32, for about 2e-7) -- for preconditioner applies only: an
 * apply precision (tdg_apply) and the multigrid smoother's (tdg_mg_opts.smooth_precision), never a
 * solve precision. */
#define TDG_FP64 0
#define TDG_FP32 1
#define TDG_MIXED 2
#define TDG_TF32 3

typedef struct tdg_op tdg_op;

/*
 * Mesh and topology as tandem's DG layer holds them:
 *  - geo_nodes: the Curvilinear geometry nodes, geo_degree warp & blend nodes per element
 *    (Curvilinear::vertices storage, src/geometry/Curvilinear.cpp:33-112), [E][Ngeo][dim];
 *  - facet_up / facet_local_no / facet_bc: FacetInfo::up, ::localNo, ::bc per local facet
 *    (src/form/FacetInfo.h:17-23, filled in src/form/DGOperatorTopo.cpp:46-85); on a boundary
 *    facet up[1] == up[0] and localNo[1] == localNo[0].
 * Element vertices must be numbered by sorted global vertex id (src/mesh/Simplex.h:15-36) so that
 * the facet quadrature points of both sides coincide.
 */
typedef struct {
    int32_t dim;            /* 2 or 3 */
    int32_t degree;         /* polynomial degree N of the DG space */
    int32_t geo_degree;     /* degree of the geometry map (tandem: Curvilinear(mesh, .., N)) */
    int32_t reserved;
    int64_t num_elements;
    int64_t num_facets;
    const double* geo_nodes;      /* [E][binom(geo_degree+dim,dim)][dim] */
    const int64_t* facet_up;      /* [F][2] */
    const int32_t* facet_local_no;/* [F][2] */
    const int32_t* facet_bc;      /* [F] */
} tdg_mesh_desc;

/*
 * Quadrature rules on the unit simplex (tandem's DGCurvilinearCommon::volRule / fctRule,
 * src/form/DGCurvilinearCommon.cpp:13-26).  fct_points has dim-1 coordinates per point.
 */
typedef struct {
    int32_t num_vol_points;
    int32_t num_fct_points;
    const double* vol_points;   /* [Nq][dim] */
    const double* vol_weights;  /* [Nq] */
    const double* fct_points;   /* [nq][dim-1] */
    const double* fct_weights;  /* [nq] */
} tdg_quadrature;

/* --- construction (replaces DGOperator's constructor and the LocalOperator prepare_* calls,
 *     src/form/DGOperator.h:54-105) ------------------------------------------------------ */

/* Builds topology and geometry (Jacobians, normals, areas, volumes) on the host. */
int tdg_create(const tdg_mesh_desc* mesh, const tdg_quadrature* quad, int kind, tdg_op** out);
void tdg_destroy(tdg_op* op);
const char* tdg_last_error(void);

/* Sizes: block size bs, Nbf, components Q, Nq, nq, E, F. */
int tdg_sizes(const tdg_op* op, int64_t out[8]);

/* Physical coordinates of the volume [E][Nq][dim] and facet [F][nq][dim] quadrature points
 * (Coords of DGCurvilinearCommon) so that the caller can evaluate its functionals there. */
int tdg_volume_coords(const tdg_op* op, double* out);
int tdg_facet_coords(const tdg_op* op, double* out);
/* Facet normals (not unit, side-0 outward) [F][nq][dim] (DGCurvilinearCommon Normal). */
int tdg_facet_normals(const tdg_op* op, double* out);

/* Material at volume quadrature points, [E][Nq] each: Poisson K (c1 unused, may be NULL),
 * Elasticity lambda and mu.  Projects onto the nodal degree-N space, evaluates the volume and
 * facet precomputations and the interior-penalty constants (Poisson::prepare_*,
 * app/localoperator/Poisson.cpp:133-223; Elasticity::prepare_*, Elasticity.cpp:104-292), then
 * uploads everything to the current device. */
int tdg_set_material(tdg_op* op, const double* c0_Q, const double* c1_Q);

/* Replaces the material as tdg_set_material does but keeps the preconditioner built for the
 * previous material (block-Jacobi inverses and the multigrid hierarchy, whichever exist), which
 * then approximates the new operator's preconditioner.  For nearby materials -- finite-difference
 * checks, line searches of an inversion -- where rebuilding the preconditioner costs more than the
 * Krylov iterations it saves (no counterpart in tandem, which rebuilds on every change).
 * TDG_E_STATE when no material or no preconditioner has been set up yet. */
int tdg_update_material(tdg_op* op, const double* c0_Q, const double* c1_Q);

/* Nodal material coefficients [E][Nbf] for c = 0, 1 (after projection). */
int tdg_material_nodal(const tdg_op* op, int c, double* out);
/* Penalty per facet [F]. */
int tdg_penalty(const tdg_op* op, double* out);

/* --- the hot path -------------------------------------------------------------------------- */

/* y = A x for nrhs stacked vectors (AbstractDGOperator::apply, src/form/AbstractDGOperator.h:34;
 * PetscDGShell::apply, app/common/PetscDGShell.cpp:48-55).  precision selects the element
 * arithmetic: TDG_FP64 takes double*, TDG_FP32 takes float*, TDG_MIXED takes double* and computes
 * in FP32 on the tensor cores (x rounded to FP32 on load, y widened on store); TDG_TF32 as
 * TDG_MIXED with one TF32 pass per product. */
int tdg_apply(tdg_op* op, int precision, const void* x, void* y, int nrhs, int64_t ld,
              void* stream);

/* y_i = A x_i for `count` independent vectors in HOST memory (x_host + i * host_stride,
 * y_host + i * host_stride; host_stride 0 = the same vector every time; double* for TDG_FP64 and
 * TDG_MIXED, float* for TDG_FP32) -- a MatMult on host-resident vectors (PetscDGShell::apply,
 * app/common/PetscDGShell.cpp:48-55, with PETSc Vecs in host memory).  Each vector is copied to
 * the device, applied and copied back; with pinned host memory the copy in of vector i + 1 and the
 * copy out of vector i - 1 overlap the apply of vector i (two device buffer pairs, three internal
 * streams, events).  Ordered after the work already on `stream`; `stream` waits for all of it.
 * Allocates the device buffers on first use and when the vectors grow. */
int tdg_apply_host(tdg_op* op, int precision, const void* x_host, void* y_host, int count, int64_t host_stride,
                   void* stream);

/* Algorithmic FLOPs and compulsory HBM bytes of one single-RHS apply (face-centric counting;
 * tandem's own count is DGOperator::flops_apply, src/form/DGOperator.h:272-280). */
int64_t tdg_flops_apply(const tdg_op* op);
int64_t tdg_bytes_apply(const tdg_op* op, int precision);

/* Block-Jacobi preconditioner (the element diagonal blocks of DGOperator::assemble,
 * src/form/DGOperator.h:121-187, applied as PETSc PCPBJACOBI would).  setup assembles the
 * diagonal blocks on the device, inverts them and stores the inverses in `precision`.
 * Returns TDG_E_NOT_SPD when a block is not positive definite. */
int tdg_bjacobi_setup(tdg_op* op, int precision, void* stream);
/* z = D^-1 r; precision is the vectors' precision: TDG_FP32 vectors need FP32 inverses, TDG_FP64
 * and TDG_MIXED (FP64 vectors) take FP64 or FP32 inverses. */
int tdg_bjacobi_apply(tdg_op* op, int precision, const void* r, void* z, int nrhs, int64_t ld,
                      void* stream);
/* Copies the assembled (not inverted) diagonal blocks [E][bs][bs] (column-major per block) to
 * host memory; for tests. */
int tdg_bjacobi_blocks(tdg_op* op, double* out);

/* --- autotuning (no counterpart in tandem) ---------------------------------------------------- */

typedef struct {
    int family;       /* 0 = element-centric tensor-core kernel, 1 = SIMT kernel, 2 = face-centric
                         tensor-core kernels (volume kernel + one pass over the facets), 3 = the
                         face-centric pair software-pipelined (FP64: asynchronous copies of the next
                         tile's coefficient blocks, tile-ordered geometry; FP32 runs family 2),
                         4 = FP32 only: family 2 with the volume term on the 5th-generation tensor
                         cores (tcgen05.mma kind::tf32, accumulators in tensor memory; shapes with at
                         most 64 volume points, else family 2) */
    int ctas_per_sm;  /* persistent CTAs per SM requested (0 = default) */
    int tile;         /* family 3, FP64: volume quadrature points per pass of the volume kernel (its
                         GEMM tiles are D x tile rows of the volume table); 0 = every point in one
                         pass where the buffers fit two CTAs per SM, else 24; other families 0 */
    double ms;        /* measured time of one apply */
} tdg_tune_entry;

/* Times the apply of this operator (its own mesh, `nrhs` right-hand sides, `precision`) for each
 * candidate launch configuration -- the tensor-core kernels (element-centric, and the
 * face-centric pair; FP64 also its software-pipelined form, FP32 also the pair with the tcgen05
 * volume kernel) at 1 to 4 persistent CTAs per SM (clipped to the occupancy limit of the
 * shape's tile), the software-pipelined FP64 form also at the tile heights that cover the volume
 * points in 1, 2, 3 and 4 passes, and the SIMT kernel -- with CUDA events on
 * `stream`, and keeps the fastest for later tdg_apply / tdg_solve calls of that precision.
 * entries (optional, up to max_entries) receives every measurement; n_entries their count. */
int tdg_autotune(tdg_op* op, int precision, int nrhs, void* stream, tdg_tune_entry* entries, int max_entries,
                 int* n_entries);
/* Sets the apply configuration of `precision` (TDG_FP64 / TDG_FP32; TDG_MIXED and TDG_TF32 follow TDG_FP32)
 * explicitly: kernel family as in tdg_tune_entry and persistent CTAs per SM. */
int tdg_set_apply_config(tdg_op* op, int precision, int family, int ctas_per_sm);
/* Sets the tile height of family 3 (TDG_FP64 only): volume points per pass of its volume kernel, as
 * tdg_tune_entry.tile; a multiple of 8 (3D) or 4 (2D), or 0 for the automatic layout.  A height whose
 * buffers do not fit the shape makes tdg_apply return TDG_E_INVALID. */
int tdg_set_apply_tile(tdg_op* op, int precision, int points_per_pass);

/* Measured FP64 throughput of the current device (no counterpart in tandem; the denominator of the
 * FP64 apply's roofline): kind 0 = FP64 FMA on the CUDA cores, 1..4 = the FP64 tensor pipe through
 * mma.sync of shape m8n8k4, m16n8k4, m16n8k8, m16n8k16, 5 = half the warps on each of the two
 * (whether they run concurrently); ctas_per_sm CTAs of 256 threads per SM
 * (0 = 2), every warp with 8 independent accumulators.  Times 3 launches of about 20 ms with CUDA
 * events on `stream` after a warm-up and returns the best rate in *tflops.  Allocates and frees
 * two small device buffers; synchronises `stream`. */
int tdg_probe_fp64_peak(int kind, int ctas_per_sm, void* stream, double* tflops);

/* Known-answer check of the 5th-generation tensor-core path of the FP32 operator (no counterpart in
 * tandem): D[128 x n] = A[128 x k] B[n x k]^T on device row-major FP32 operands through tcgen05.mma
 * kind::tf32 with the accumulator in tensor memory, in three TF32 products (hi hi + hi lo + lo hi)
 * when split3 = 1, one when 0; both operands K-major in shared memory (core matrices of 8 rows x
 * 16 bytes).  n a multiple of 16 in [16, 256], k a multiple of 8 in [8, 64].  Synchronises `stream`;
 * TDG_E_TIMEOUT when the MMA's completion was not seen within the bounded wait (about 2 s of wall
 * clock); split3 = -1 issues no MMA and no commit, so that the wait runs out and the error path
 * (status word, tensor memory freed, TDG_E_TIMEOUT) can be tested. */
int tdg_probe_tc05_gemm(const float* A, const float* B, float* D, int n, int k, int split3, void* stream);
/* The accumulator layout of a tcgen05 kind::tf32 MMA (no counterpart in tandem): D = A[m x k]
 * B[n x k]^T in three TF32 products for m = 64 or 128, then every tensor-memory lane 0..127 and
 * columns 0..2n-1 (pre-filled with -12345) copied to dump[128][2n].  n a multiple of 16 in [16, 128],
 * k a multiple of 8 in [8, 64].  Synchronises `stream`. */
int tdg_probe_tc05_layout(const float* A, const float* B, float* dump, int m, int n, int k, void* stream);

/* --- right-hand side (DGOperator::rhs, src/form/DGOperator.h:189-237) ---------------------- */

/* b = volume load + boundary/fault lift terms.  force_Q: [E][Q][Nq] at volume points (may be
 * NULL); bc_q: [F][Q][nq] Dirichlet or slip data at facet points (may be NULL), given exactly as
 * tandem's facet functional returns it for the facet (sign already oriented).  Host arrays in,
 * host array out [E][bs]. */
int tdg_rhs(tdg_op* op, const double* force_Q, const double* bc_q, double* b);

/* --- Krylov solve on the device (PetscLinearSolver / KSPCG, app/common/PetscLinearSolver.cpp) */

typedef struct {
    int32_t precision;      /* TDG_FP64: FP64 CG.  TDG_MIXED: FP64 CG recurrence around the FP32
                               operator, with the block inverses of the last tdg_bjacobi_setup
                               (FP32 or FP64).  TDG_FP32: FP32 CG
                               recurrence and vectors.  Both reduced-precision modes keep the
                               solution and the true residual in FP64 (reliable updates); problems
                               whose TDG_FP32 recurrence stalls above the target continue in FP64 */
    int32_t max_iterations; /* total Krylov iterations cap */
    double rtol;            /* relative residual ||b - A x|| / ||b|| target (FP64 residual) */
    double inner_rtol;      /* reliable-update threshold: the FP64 residual replaces the recurrence
                               residual whenever the latter has dropped by this factor
                               (0 = default: 0.1) */
    int32_t max_outer;      /* cap on reliable updates (0 = none) */
    int32_t use_graphs;     /* capture iteration blocks in CUDA graphs (needs a non-NULL stream):
                               each block is a device loop (a conditional while node) that ends
                               at the iteration where a problem's recurrence residual asks for a
                               reliable update, or after 32 iterations; the host reads the
                               scalars between blocks.  0: the host launches every iteration and
                               checks every 8 (every one under multigrid) */
    int32_t method;         /* TDG_KSP_CG (default) or TDG_KSP_FGMRES */
    int32_t restart;        /* FGMRES restart length m (0 = 30; at most 64) */
} tdg_solve_opts;

/* Krylov methods of tdg_solve / tdg_solve_segmented (KSPCG, and KSPFGMRES as tandem's multigrid
 * configuration selects it, examples/options/mg_cheby.cfg:2).  TDG_KSP_FGMRES: restarted flexible
 * GMRES(m) with right preconditioning, FP64 vectors, one Arnoldi process per right-hand side or
 * problem; classical Gram-Schmidt applied twice, each pass one batched multi-dot reduction; every
 * cycle starts from the FP64 residual b - A x.  Precision TDG_FP64 or TDG_MIXED (the operator and
 * the preconditioner in FP32 arithmetic inside the FP64 cycles).  In tdg_solve_stats, iterations
 * counts Arnoldi steps and outer the restart cycles. */
#define TDG_KSP_CG 0
#define TDG_KSP_FGMRES 1

typedef struct {
    int32_t iterations;     /* total Krylov iterations */
    int32_t outer;          /* reliable updates (FP64 residual replacements) */
    double rel_residual;    /* final FP64 relative residual */
    double seconds;         /* device time of the solve */
    int32_t converged;
    int32_t fp64_iterations; /* mixed: iterations of the FP64 continuation (0 if none) */
} tdg_solve_stats;

/* Solves A x = b (device double arrays, nrhs stacked with leading dimension ld) with
 * preconditioned CG (reliable updates: the recurrence residual is periodically replaced by the
 * FP64 residual b - A x, keeping the search direction).  x holds the initial guess.  The
 * preconditioner is the one tdg_set_preconditioner selected: block Jacobi (default;
 * tdg_bjacobi_setup must have been called with the precision the solve needs, FP64 for TDG_FP64,
 * FP32 for TDG_FP32) or the multigrid V-cycle (tdg_mg_setup; TDG_FP64 or TDG_MIXED; flexible CG). */
int tdg_solve(tdg_op* op, const double* b, double* x, int nrhs, int64_t ld,
              const tdg_solve_opts* opts, tdg_solve_stats* stats, void* stream);

/* Solves a block-diagonal batch of independent problems held in one operator (the disjoint union
 * of several meshes): segment s owns elements [seg_elem_offset[s], seg_elem_offset[s+1]) (host
 * array, nseg + 1 entries, covering [0, E)) and gets its own Krylov scalars and convergence test,
 * while every apply and preconditioner launch covers all problems at once.
 * seg_rel_residual (host, may be NULL) receives each problem's final relative residual. */
int tdg_solve_segmented(tdg_op* op, const double* b, double* x, int nseg, const int64_t* seg_elem_offset,
                        const tdg_solve_opts* opts, tdg_solve_stats* stats, double* seg_rel_residual,
                        void* stream);

/* One rank's part of a solve over a distributed operator (tandem's MPI distribution of
 * DGOperator, src/form/DGOperator.h:382-393, with PETSc's parallel KSPCG): `op` is the rank's local
 * operator -- its owned elements first, then one layer of ghost elements -- and b, x are local device
 * vectors of E * bs entries whose first owned_elements * bs rows are this rank's part of the global
 * vectors.  CG with the block-Jacobi preconditioner of the local operator (tdg_bjacobi_setup) runs
 * on the owned rows; before every apply the library calls exchange(ctx, v, stream), which must fill
 * the ghost blocks of the device vector v with the owning ranks' values, and after every local
 * reduction allreduce(ctx, values, count, stream), which must replace the `count` device doubles
 * at `values` by their sums over the ranks.  Both are expected to enqueue their work on `stream`
 * (e.g. NCCL point-to-point and all-reduce) and return 0; every rank calls them in the same order
 * (two all-reduces per iteration, plus two per reliable update).  TDG_FP64 or TDG_MIXED, method
 * TDG_KSP_CG; no CUDA graphs (the callbacks run on the host).  The stopping test uses the global
 * FP64 residual. */
typedef int (*tdg_exchange_fn)(void* ctx, double* v, void* stream);
typedef int (*tdg_allreduce_fn)(void* ctx, double* values, int count, void* stream);
int tdg_solve_distributed(tdg_op* op, const double* b, double* x, int64_t owned_elements,
                          const tdg_solve_opts* opts, tdg_solve_stats* stats, tdg_exchange_fn exchange,
                          tdg_allreduce_fn allreduce, void* ctx, void* stream);

/* --- p-multigrid preconditioner (PetscLinearSolver::setup_mg, app/common/PetscLinearSolver.cpp:53-114,
 *     MGConfig, app/common/MGConfig.cpp:11-41, options examples/options/mg_cheby.cfg) ------------ */

#define TDG_PC_BJACOBI 0
#define TDG_PC_MG 1

#define TDG_MG_TWOLEVEL 0
#define TDG_MG_LOGARITHMIC 1
#define TDG_MG_FULL 2

#define TDG_MG_COARSE_DG 0
#define TDG_MG_COARSE_P1 1

typedef struct {
    int32_t strategy;        /* TDG_MG_TWOLEVEL / LOGARITHMIC / FULL (MGStrategy; default logarithmic) */
    int32_t coarse_degree;   /* degree of the coarsest level (MGConfig coarse_level; default 1) */
    int32_t smooth_its;      /* Chebyshev steps per smoothing (-mg_levels_ksp_max_it; default 10) */
    double esteig_lo;        /* smoothing interval [esteig_lo, esteig_hi] x lambda_max(D^-1 A)   */
    double esteig_hi;        /* (-mg_levels_ksp_chebyshev_esteig 0,lo,0,hi; default 0.01, 1.1)    */
    int32_t esteig_steps;    /* Lanczos steps of the lambda_max estimate (default 10) */
    double coarse_rtol;      /* coarsest-level CG relative tolerance (-mg_coarse_ksp_rtol; 0.1) */
    int32_t coarse_max_it;   /* coarsest-level CG iteration cap (default 1000) */
    int32_t smooth_precision; /* TDG_FP64, or TDG_MIXED: FP32 arithmetic for the finest level's
                                 smoother applies, FP32 copies of the blocks for the smoothed levels
                                 below it (vectors, accumulation and the coarse solve stay FP64);
                                 TDG_TF32: the same with the finest level's smoother applies in one
                                 TF32 pass (the solve's own operator keeps its precision) */
    int32_t coarse_space;    /* TDG_MG_COARSE_DG: the coarse CG works on the coarsest DG level (as
                                tandem's -mg_coarse_ksp_type cg).  TDG_MG_COARSE_P1 (default): the
                                coarsest DG level is smoothed too and corrected from the continuous
                                P1 space on the mesh vertices (Galerkin R^T A R, rigid-body modes
                                included), where the coarse CG runs -- in place of tandem's GAMG */
} tdg_mg_opts;

/* Builds the p-multigrid hierarchy: level degrees from the strategy; the element interpolation
 * between consecutive degrees (modal injection for Poisson, nodal interpolation for elasticity,
 * ModalInterpolation.h:40-44, NodalInterpolation.cpp:8-36); Galerkin coarse operators
 * A_l = I^T A_{l+1} I (the first by probing the matrix-free operator with a distance-2 element
 * colouring, the others by block triple products) stored element block-sparse on the device;
 * point-Jacobi diagonals; the lambda_max estimates of the Chebyshev smoothers; the coarse system
 * (see coarse_space) with its block-Jacobi inverses.  opts may be NULL (defaults: logarithmic,
 * coarse degree 1, continuous P1 coarse space).  Does not select the preconditioner
 * (tdg_set_preconditioner).  tdg_set_material invalidates the hierarchy (as it does the
 * block-Jacobi inverses): call tdg_mg_setup again before the next multigrid solve. */
int tdg_mg_setup(tdg_op* op, const tdg_mg_opts* opts, void* stream);
/* z = M r, one V-cycle per right-hand side (PCMG's apply): Chebyshev pre-smoothing from zero,
 * restriction of the residual, the coarser levels, prolongation, Chebyshev post-smoothing; CG with
 * block Jacobi on the coarsest level.  FP64 device vectors.  The coarse CG runs as a device loop
 * (a CUDA graph with a conditional while node, its stopping test on the device every 8
 * iterations), so the V-cycle itself never waits for the host; the call then synchronises `stream`
 * to report a coarse CG whose residual became non-finite (TDG_E_DIVERGED). */
int tdg_mg_apply(tdg_op* op, const double* r, double* z, int nrhs, int64_t ld, void* stream);
/* Preconditioner of tdg_solve / tdg_solve_segmented (and the Green's-function and adjoint solves
 * built on them): TDG_PC_BJACOBI (default) or TDG_PC_MG (needs tdg_mg_setup; TDG_FP64 and
 * TDG_MIXED solves; the Krylov method becomes flexible CG, since the coarse CG makes the
 * preconditioner vary slightly between iterations). */
int tdg_set_preconditioner(tdg_op* op, int pc);
/* Hierarchy description: number of levels; per level (coarsest first, up to max_levels) the
 * degree, block size and lambda_max estimate (the finest level's too; level 0 has none: 0).
 * Any output may be NULL.  coarse_its: coarsest-level CG iterations since setup (may be NULL). */
int tdg_mg_info(tdg_op* op, int* nlevels, int max_levels, int* degrees, int* block_sizes, double* lambda_max,
                int64_t* coarse_its);
/* Copies level `level` (< nlevels - 1) of the hierarchy to host memory: blocks [E][NB][bs][bs]
 * (column-major per block, NB = 1 + faces per element) and its neighbour table nbr [E][NB]
 * (slot 0 the element, slot 1 + f the element behind face f, -1 none); for tests. */
int tdg_mg_level_matrix(tdg_op* op, int level, double* blocks, int32_t* nbr);
/* Host utilities (no device): the level degrees of a strategy (returns their count; degrees may
 * be NULL) and the reference interpolation matrix [Nbf(n_to)][Nbf(n_from)] of one component. */
int tdg_mg_level_degrees(int strategy, int coarse_degree, int degree, int* degrees);
int tdg_mg_interpolation(int dim, int kind, int n_to, int n_from, double* out);
/* Host utilities of an operator (no device work, no tdg_set_material needed):
 * the element colouring the Galerkin probing uses (distance 2 across interior facets: an element's
 * neighbours and their neighbours all differ from it), colour [E], *ncolours;
 * the vertex numbering of the continuous P1 coarse space (corners identified across interior
 * facets only), vid [E][dim + 1] in the element's corner order, *nv. */
int tdg_mg_colouring(const tdg_op* op, int32_t* colour, int* ncolours);
/* The continuous P1 coarse space's element embedding (host only): out [Nbf(degree)][dim + 1], the
 * coefficients in the degree-`degree` space of `kind` (modal for TDG_POISSON, nodal for
 * TDG_ELASTICITY) of the linear function that is 1 at corner i and 0 at the other corners. */
int tdg_mg_p1_embedding(int dim, int kind, int degree, double* out);
int tdg_mg_vertex_numbering(const tdg_op* op, int32_t* vid, int64_t* nv);

/* --- explicit wave operator (Elasticity::wave_rhs, app/localoperator/Elasticity.cpp:865-880) -- */

/* Density rho at the volume points [E][Nq] (Elasticity's optional rho functional,
 * Elasticity.cpp:28-35; 1/rho is projected onto the nodal material space like lam and mu).
 * Default rho = 1.  Elasticity only. */
int tdg_set_density(tdg_op* op, const double* rho_Q);
/* y = -(1/rho)-weighted inverse mass applied to x (tandem's apply_inverse_mass kernel,
 * app/kernels/elasticity.py:236-237: the reference inverse mass with -rhoInv W / |J| at the volume
 * points); device FP64 arrays, nrhs stacked with leading dimension ld; y may alias x. */
int tdg_apply_inverse_mass(tdg_op* op, const double* x, double* y, int nrhs, int64_t ld, void* stream);
/* y = wave_rhs(x) = inverse mass applied to (A x - b): the acceleration of rho u'' = b - A u.  b is
 * the boundary / slip data part of the right-hand side at the current time (tdg_rhs with only
 * bc_q, uploaded; tandem adds the same data inside the fluxes), or NULL for none.  y must not
 * alias x or b. */
int tdg_wave_rhs(tdg_op* op, const double* x, const double* b, double* y, int nrhs, int64_t ld, void* stream);

/* --- adjoint gradient (no counterpart in tandem: tandem solves forward problems only) ---------- */

/* Gradient of a functional J(u) with respect to per-element constant Lame parameters of an
 * elasticity operator whose material is piecewise constant (lambda_e, mu_e per element):
 * grad[e][0] = dJ/dlambda_e, grad[e][1] = dJ/dmu_e = p^T db/dtheta_e - p^T dA/dtheta_e u, where u
 * solves A u = b and p solves A p = dJ/du (A is symmetric).  u, p: device [E][bs]; bc_q: device
 * [F][D][nq] Dirichlet / slip data used in b (NULL when b has no boundary data); grad: device
 * [E][2].  TDG_E_INVALID when the material is not piecewise constant. */
int tdg_adjoint_lame_gradient(tdg_op* op, const double* u, const double* p, const double* bc_q, double* grad,
                              void* stream);

/* Allocation-free variant of tdg_adjoint_lame_gradient (no counterpart in tandem).  Same inputs,
 * output and arithmetic; on success it calls no device or host allocator.  For callers that cannot
 * allocate device memory at the time of the call: a process whose caching allocator (torch, PETSc
 * pools) already holds the device memory, where a fresh cudaMallocAsync can fail with out-of-memory
 * in the middle of an optimisation loop, or a caller running inside an allocator or memory-pool
 * callback.  The per-facet penalty derivatives go through a fixed device scratch, a static
 * __device__ array of 2^20 doubles (8 MiB) per device, staged from a static host buffer of 2^16
 * doubles: meshes with 4 F + 2 E > 2^20 (about 120,000 tetrahedra or 170,000 triangles) return
 * TDG_E_INVALID with the sizes in tdg_last_error.  Every scratch entry the kernel reads is written
 * by the call, so nothing needs clearing.  The operator's FP64 data must already be resident (one
 * FP64 tdg_apply after tdg_set_material), else TDG_E_STATE: that upload, on the device current at
 * the time, also looks up the scratch address (cudaGetSymbolAddress) and loads the gradient kernel,
 * the two steps that can place the scratch or code in device memory, so this call itself does
 * neither.  Calls on one device share the scratch (and all calls the host buffer): overlapping
 * calls (two host threads, or two streams) race on the device and must be serialised by the
 * caller.  The call synchronises `stream` before returning.  A failing call records its message
 * for tdg_last_error in a thread-local string, which may allocate host memory. */
int tdg_adjoint_lame_gradient_noalloc(tdg_op* op, const double* u, const double* p, const double* bc_q,
                                      double* grad, void* stream);

/* --- fault coupling, Green's functions (app/form/SeasQDDiscreteGreenOperator.cpp:493-578) ---- */

typedef struct tdg_fault tdg_fault;

/* Prepares the fault facets as tandem's AdapterBase::prepare does
 * (app/localoperator/AdapterBase.cpp:44-99): oriented facet normals (flipped where they point
 * against ref_normal), fault mass matrices of the nodal degree-N fault basis and their inverses.
 * fault_facets lists facet numbers (BoundaryMap order).  Poisson operators only; the operator must
 * outlive the fault object. */
int tdg_fault_create(tdg_op* op, int64_t num_fault, const int64_t* fault_facets, const double* ref_normal,
                     tdg_fault** out);
void tdg_fault_destroy(tdg_fault* fault);
/* out[0] = fault facets, out[1] = fault basis functions per facet. */
int tdg_fault_sizes(const tdg_fault* fault, int64_t out[2]);
/* b += right-hand side of the slip (Adapter::slip + Poisson::rhs_skeleton/boundary).  slip:
 * device [nrhs][ld_slip] with ld_slip >= num_fault * nbf; b: device [nrhs][ld]. */
int tdg_fault_slip_rhs(tdg_fault* fault, const double* slip, int64_t ld_slip, double* b, int nrhs, int64_t ld,
                       void* stream);
/* traction = fault-basis traction of (u, slip) (Poisson::traction_skeleton/boundary +
 * Adapter<Poisson>::traction).  u: device [nrhs][ld]; slip may be NULL (zero slip); traction:
 * device [nrhs][ld_t] with ld_t >= num_fault * nbf. */
int tdg_fault_traction(tdg_fault* fault, const double* u, int64_t ld, const double* slip, int64_t ld_slip,
                       double* traction, int64_t ld_t, int nrhs, void* stream);

/* Traction update of the discrete Green's function operator
 * (SeasQDDiscreteGreenOperator::update_traction, app/form/SeasQDDiscreteGreenOperator.cpp:115-127:
 * MatMult(G_, S, traction) followed by VecAXPY(traction, time, t_boundary_)) in one kernel, for k
 * slip states at once: out[j * ldo + i] = sum_c G[i * ldg + c] S[j * lds + c] + time t_boundary[i],
 * i < n, c < m, j < k.  G: device, dense row-major n x m (leading dimension ldg >= m), read once
 * per group of 4 states; S: device [k][lds]; t_boundary: device [n] or NULL (no boundary term);
 * out: device [k][ldo], must not overlap S.  m <= 7264 (the states of a group sit in shared
 * memory). */
int tdg_gf_traction_update(int64_t n, int64_t m, const double* G, int64_t ldg, const double* S, int64_t lds,
                           int k, const double* t_boundary, double time, double* out, int64_t ldo, void* stream);

/* --- projection and evaluation (host; AbstractDGOperator::project / solution) -------------------- */

/* y [E][bs] = the projection of values at the volume points U_Q [E][Q][Nq] (Elasticity::project,
 * app/localoperator/Elasticity.cpp:882-911: weight-adjusted inverse mass of E_Q W |J| U_Q; exact
 * for the discrete space on affine elements; here for both kinds). */
int tdg_project(const tdg_op* op, const double* U_Q, double* y);
/* The discrete function x [E][bs] (host) at np unit-simplex points [np][dim] of every element:
 * out [E][Q][np] (DGOperator::solution + FiniteElementFunction::map). */
int tdg_evaluate(const tdg_op* op, const double* x, int np, const double* points, double* out);

/* --- error norms (Error<D>::L2 / H1_semi, src/form/Error.cpp; host post-processing) ---------- */

/* tandem integrates the error with its own rule (simplexQuadratureRule<D>(20)); the caller passes
 * the rule here: np points on the unit simplex [np][dim] and weights [np] (tdg_conical_rule gives
 * tandem's conical product rules).  tdg_rule_coords maps the points to every element, out
 * [E][np][dim], for the caller to evaluate its reference solution there.  x: the solution on the
 * host [E][bs].  ref: reference values [E][Q][np]; refgrad: reference physical gradients
 * [E][Q][dim][np].  *out: the norm (square root of the summed integrals). */
int tdg_rule_coords(const tdg_op* op, int np, const double* points, double* out);
int tdg_error_l2(const tdg_op* op, const double* x, int np, const double* points, const double* weights,
                 const double* ref, double* out);
int tdg_error_h1_semi(const tdg_op* op, const double* x, int np, const double* points, const double* weights,
                      const double* refgrad, double* out);

/* --- host utilities: reference-element tables (no device work) ---------------------------- */

/* Reference nodes of degree N on the unit simplex: family 0 = warp & blend
 * (src/basis/WarpAndBlend.cpp), 1 = equidistant in VTK order (src/basis/Equidistant.cpp).
 * out: [binom(N+dim,dim)][dim]. */
int tdg_ref_nodes(int dim, int degree, int family, double* out);
/* Basis of degree N at np points: family -1 = modal Dubiner (src/basis/Functions.cpp), 0/1 =
 * nodal Lagrange basis at the warp & blend / equidistant nodes.  E: [Nbf][np] (may be NULL),
 * grad: [Nbf][dim][np] (may be NULL). */
int tdg_ref_basis(int dim, int degree, int family, int np, const double* points, double* E, double* grad);
/* Conical Gauss-Jacobi product rule of at least `order` on the unit simplex
 * (src/quadrules/TensorProductRule.cpp); returns the number of points, fills points/weights when
 * non-NULL. */
int tdg_conical_rule(int dim, int order, double* points, double* weights);

#ifdef __cplusplus
}
#endif

#endif /* TANDEM_B200_H */
