// Host-side operator set-up: topology, curvilinear geometry at quadrature points, material
// projection, facet coefficients and interior-penalty constants.  Produces flat arrays that the
// device layer uploads unchanged; the device kernels only ever read these arrays.
#pragma once

#include "refelem.hpp"

#include <cstdint>
#include <vector>

namespace tdg {

// Per element and local face: the view of one facet from one of its elements (tandem's
// SideInfo, src/form/FacetInfo.h:11-17).  nb == element itself on a boundary facet.
struct Side {
    int32_t fct;
    int32_t side;      // 0 or 1: which FacetInfo side the element is
    int32_t nb;        // element on the other side
    int32_t nb_local;  // local face number of the facet in nb
    int32_t bc;
};

struct HostOperator {
    // sizes
    int D = 0, N = 0, kind = 0;
    int Nbf = 0, Q = 0, bs = 0, Nq = 0, nq = 0, nfaces = 0, geoN = 0, Ngeo = 0;
    int64_t E = 0, F = 0;

    // quadrature
    Points vol_x, fct_x;          // unit simplex / unit facet coordinates
    std::vector<double> W, w;     // weights

    // solution space tables (modal for Poisson, nodal warp & blend for Elasticity)
    RefSpace space, mat_space, geo_space;
    Dense E_Q;                    // [Nbf][Nq]
    std::vector<double> Dxi_Q;    // [Nbf][D][Nq]
    std::vector<Dense> E_qf;      // per local face: [Nbf][nq]
    std::vector<std::vector<double>> Dxi_qf;  // per local face: [Nbf][D][nq]
    Dense matE_Q;                 // [Nbf][Nq] material (nodal) basis
    std::vector<Dense> matE_qf;   // per local face [Nbf][nq]

    // topology
    std::vector<int64_t> up;      // [F][2]
    std::vector<int32_t> loc;     // [F][2]
    std::vector<int32_t> bc;      // [F]
    std::vector<Side> sides;      // [E][nfaces]

    // geometry (reference layout: G(e, i) = d xi_e / d x_i at each point)
    std::vector<double> geo_nodes;   // [E][Ngeo][D]
    std::vector<double> vG;          // [E][D*D][Nq]  index (e*D+i)
    std::vector<double> vAbsDetJ;    // [E][Nq]
    std::vector<double> vCoords;     // [E][Nq][D]
    std::vector<double> volume;      // [E]
    std::vector<double> fN;          // [F][D][nq] normal (side 0 outward, |detJ| scaled)
    std::vector<double> fNunit;      // [F][D][nq]
    std::vector<double> fNl;         // [F][nq]
    std::vector<double> fG0, fG1;    // [F][D*D][nq]
    std::vector<double> fCoords;     // [F][nq][D]
    std::vector<double> area;        // [F]

    // material (after tdg_set_material)
    bool has_material = false;
    std::vector<double> mat_nodal;   // [E][2][Nbf]  (Poisson: K, 0; Elasticity: lam, mu)
    std::vector<double> vCoef;       // [E][ncoef][Nq]  Poisson: J*W*K; Elasticity: lam*W*J, mu*W*J
    int ncoef = 0;
    std::vector<double> fCoef;       // Poisson: [F][2][D*D][nq] K*G0, K*G1
                                     // Elasticity: [F][4][nq] lam0, mu0, lam1, mu1
    std::vector<double> penalty;     // [F]

    void build(int D, int N, int geoN, int kind, int64_t E, int64_t F, double const* geo_nodes,
               int64_t const* facet_up, int32_t const* facet_loc, int32_t const* facet_bc,
               int nvol, double const* vol_x, double const* vol_w, int nfct, double const* fct_x,
               double const* fct_w);
    void set_material(double const* c0_Q, double const* c1_Q);

    // Explicit wave operator (Elasticity::wave_rhs, app/localoperator/Elasticity.cpp:865-880):
    // Minv_ref = inverse of the reference mass matrix, nrwj[E][Nq] = -rhoInv(x_q) W_q / |J|_q
    // (negative_rhoInv_W_Jinv_Q, app/kernels/elasticity.py:44-48), rho = 1 until set_density.
    Dense Minv_ref;
    std::vector<double> nrwj;
    void set_density(double const* rho_Q);
    void default_density();

    // Diagonal blocks of the assembled operator, [E][bs][bs] column-major per block
    // (DGOperator::assemble restricted to A(e, e)).  Host reference used by tests and as the
    // fallback-free source of truth for the device assembly kernel's layout.
    void rhs(double const* force_Q, double const* bc_q, double* b) const;

    int64_t flops_apply() const;
    int64_t bytes_apply(int scalar_bytes) const;

    // Error<D>::L2 / H1_semi (src/form/Error.cpp:13-48, 120-170) of the solution x [E][bs] against a
    // reference given at the np points (unit simplex, [np][D]) of a caller-chosen rule with weights
    // w (tandem integrates with simplexQuadratureRule<D>(20)): ref [E][Q][np] values, refgrad
    // [E][Q][D][np] physical gradients.  rule_coords: the points mapped to every element, out
    // [E][np][D], where the caller evaluates its reference.
    void rule_coords(int np, double const* pts, double* out) const;

    // Elasticity::project (app/localoperator/Elasticity.cpp:882-911): y [E][bs] from values at the
    // volume points U_Q [E][Q][Nq]: the weight-adjusted inverse mass (kernel apply_inverse_mass
    // with weights W/|J|, app/kernels/elasticity.py:236-237) of E_Q W |J| U_Q (project_u_rhs);
    // exact for the discrete space on affine elements.  Offered for both kinds.
    void project(double const* U_Q, double* y) const;
    // The discrete function x [E][bs] at unit-simplex points pts [np][D] of every element, out
    // [E][Q][np] (FiniteElementFunction::map over DGOperator::solution).
    void evaluate(double const* x, int np, double const* pts, double* out) const;
    double error_l2(double const* x, int np, double const* pts, double const* w, double const* ref) const;
    double error_h1_semi(double const* x, int np, double const* pts, double const* w, double const* refgrad) const;
};

// ---- p-multigrid set-up (tandem's PCMG path, app/common/PetscLinearSolver.cpp:53-114) ----------

// Reference interpolation from degree n_from to degree n_to > n_from, [Nbf(n_to)][Nbf(n_from)]
// per component (the element interpolation is block diagonal over components).  Modal spaces
// (Poisson): injection of the first Nbf(n_from) Dubiner coefficients (ModalInterpolation.h:40-44).
// Nodal spaces (Elasticity): the coarse Lagrange basis at the fine warp & blend nodes, which is
// V_to[:, :N2] V_from^-1 (NodalInterpolation.cpp:8-36).  Both embed the coarse space exactly.
Dense interpolation_matrix(int D, int kind, int n_to, int n_from);

// Polynomial degrees of the levels, coarsest first (MGConfig::levels, app/common/MGConfig.cpp:11-41):
// strategy 0 two-level {coarse, N}; 1 logarithmic (N, N/2, ... down to coarse); 2 full
// (coarse, coarse+1, ..., N).  A coarse degree >= N becomes N - 1.
std::vector<int> mg_level_degrees(int strategy, int coarse, int N);

// Element neighbours across interior facets: nbr[e][0] = e, nbr[e][1 + f] = the element behind
// local face f, or -1 on a boundary facet (whose coupling is part of the element's own block).
std::vector<int32_t> element_neighbours(HostOperator const& h);

// Greedy distance-2 colouring of the element graph: two elements that share a facet or a
// neighbour get different colours, so every element's closed neighbourhood holds each colour at
// most once.  Returns the colour per element and sets ncolors.
std::vector<int32_t> distance2_colouring(std::vector<int32_t> const& nbr, int64_t E, int NB, int* ncolors);

// ---- continuous P1 auxiliary coarse space (below the coarsest DG level) ---------------------------

// Global vertex numbers vid[e][i] of the element corners, from the facet connectivity alone: the
// corners of a facet are identified across its two elements (both list a facet's corners in the
// same order, as element corners are sorted by global id), so vertices are shared exactly within
// facet-connected parts of the mesh (independent problems of a mesh union stay apart).
std::vector<int32_t> vertex_numbering(HostOperator const& h, int64_t* nv);

// T [Nbf(p)][D+1]: coefficients in the operator's degree-p space (modal Dubiner or nodal warp &
// blend) of the linear function with value 1 at corner i and 0 at the others.
Dense linear_to_space(int D, int kind, int p);

// Galerkin operator R^T A R of the continuous P1 space for the element block-sparse matrix A
// [E][NB][bs][bs] (column-major blocks, bs = Nbf(p) Q), R_e = T per component on element e's
// corners.  Rows of Q x Q blocks by vertex, CSR: ptr [nv + 1], col [nnzb], val [nnzb][Q][Q]
// (row-major).  vinc_ptr/vinc: the (element, corner) incidences of each vertex (e * (D+1) + i).
struct VertexCsr {
    int64_t nv = 0;
    int Q = 0;
    std::vector<int64_t> ptr;
    std::vector<int32_t> col;
    std::vector<double> val;
    std::vector<int64_t> vinc_ptr;
    std::vector<int32_t> vinc;
};
VertexCsr vertex_galerkin(std::vector<double> const& A, std::vector<int32_t> const& nbr, int64_t E, int NB, int D,
                          int Nbf, int Q, Dense const& T, std::vector<int32_t> const& vid, int64_t nv);

}  // namespace tdg
