// Reference-element tables for degree-N simplices: multi-index enumeration, Jacobi and Dubiner
// polynomials, Gauss-Jacobi rules, warp & blend and equidistant nodes, Vandermonde matrices and
// basis evaluation.  Setup-time host code; every table the device kernels read is built here.
//
// The enumeration orders (basis functions, nodes, facet-to-vertex maps) must agree with tandem's,
// because they define the layout of the solution vectors handed across the C ABI.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace tdg {

// Points on a D-simplex are stored flat: point p, coordinate d at [p * D + d].
using Points = std::vector<double>;

// Dense row-major matrix.
struct Dense {
    int rows = 0, cols = 0;
    std::vector<double> a;
    Dense() = default;
    Dense(int r, int c) : rows(r), cols(c), a(static_cast<std::size_t>(r) * c, 0.0) {}
    double& operator()(int i, int j) { return a[static_cast<std::size_t>(i) * cols + j]; }
    double operator()(int i, int j) const { return a[static_cast<std::size_t>(i) * cols + j]; }
};

// Inverse by Gauss-Jordan elimination with partial pivoting; throws on a singular matrix.
Dense invert(Dense const& m);
// Solves m x = b in place (b has m.rows entries), LU with partial pivoting.
void solve_in_place(Dense m, double* b);

inline std::size_t binom(unsigned n, unsigned k) {
    std::size_t r = 1;
    for (unsigned i = 1; i <= k; ++i) {
        r = r * (n - k + i) / i;
    }
    return r;
}
inline int num_basis(int D, int N) { return static_cast<int>(binom(N + D, D)); }

// Multi-indices j with |j| <= N in tandem's enumeration order (AllIntegerSums,
// src/util/Combinatorics.h:47-115): graded by total degree; the first entry decreases fastest.
// Each entry holds D valid components.
std::vector<std::array<unsigned, 3>> graded_multi_indices(int D, unsigned N);

// Jacobi polynomial P_n^{(a,b)}(x) by the three-term recurrence (src/basis/Functions.cpp:6-23).
double jacobi_p(unsigned n, unsigned a, unsigned b, double x);
double jacobi_p_derivative(unsigned n, unsigned a, unsigned b, double x);
// Homogenised ("singularity free") Jacobi polynomial y^n P_n^{(a,b)}(x/y) and its partial
// derivatives in x and y (src/basis/Functions.cpp:25-88).
double sf_jacobi_p(unsigned n, unsigned a, unsigned b, double x, double y);
std::array<double, 3> sf_jacobi_p_and_derivatives(unsigned n, unsigned a, unsigned b, double x,
                                                  double y);

// Unnormalised Dubiner polynomials on the unit simplex (src/basis/Functions.cpp:90-151).
double dubiner(int D, std::array<unsigned, 3> const& j, double const* xi);
std::array<double, 3> grad_dubiner(int D, std::array<unsigned, 3> const& j, double const* xi);

// Gauss-Jacobi rule with weight (1-x)^a (1+x)^b on [-1,1] (src/quadrules/GaussJacobi.cpp:13-38).
struct IntervalRule {
    std::vector<double> x, w;
};
IntervalRule gauss_jacobi(unsigned n, unsigned a, unsigned b);
// Legendre-Gauss-Lobatto points on [-1,1] (src/basis/Nodal.cpp:17-27).
std::vector<double> lgl_points(unsigned n);

// Quadrature rule on the unit simplex {x_i >= 0, sum x_i <= 1}.
struct SimplexRule {
    int dim = 0;
    int order = 0;
    Points x;
    std::vector<double> w;
    int size() const { return static_cast<int>(w.size()); }
};
// Conical (collapsed) Gauss-Jacobi product rule with n = 1 + order/2 points per direction
// (src/quadrules/TensorProductRule.cpp:10-75).  For D = 1 it is the Gauss-Legendre rule tandem
// uses on every facet of a triangle mesh.
SimplexRule conical_product_rule(int D, unsigned min_order);

// Warp & blend nodes of degree N on the unit simplex, D = 1, 2, 3
// (src/basis/WarpAndBlend.cpp; Hesthaven & Warburton, Nodal DG methods, 2008).
Points warp_blend_nodes(int D, unsigned N);
// Equidistant nodes in VTK ordering (src/basis/Equidistant.cpp), D = 2, 3.
Points equidistant_nodes(int D, unsigned N);

// Vandermonde matrix V(i, j) = Dubiner_j(node_i) (src/basis/Nodal.cpp:29-43).
Dense vandermonde(int D, unsigned N, Points const& nodes);

// Function space on the reference simplex: modal (Dubiner) or nodal (Lagrange at `nodes`).
class RefSpace {
public:
    static RefSpace modal(int D, unsigned N);
    static RefSpace nodal(int D, unsigned N, Points nodes);

    int dim() const { return D_; }
    int degree() const { return N_; }
    int num_basis() const { return nbf_; }
    bool is_nodal() const { return nodal_; }
    Points const& nodes() const { return nodes_; }

    // E(k, q): basis function k at point q.
    Dense eval(Points const& pts) const;
    // G[(k * D + d) * np + q]: d-th reference derivative of basis function k at point q.
    std::vector<double> grad(Points const& pts) const;
    // Reference mass matrix (modal: diagonal, computed with a degree-2N rule; nodal: V^-T M V^-1).
    Dense mass_matrix() const;

private:
    int D_ = 0, N_ = 0, nbf_ = 0;
    bool nodal_ = false;
    Points nodes_;
    Dense Vinv_;  // inverse Vandermonde (nodal only)
    std::vector<std::array<unsigned, 3>> idx_;
};

// Facet-to-vertex map of the reference simplex: facet f of the unit D-simplex has vertices
// facet_vertices(D)[f] (k-subsets in lexicographic order, src/mesh/Simplex.h:86-108).
std::vector<std::array<int, 3>> facet_vertices(int D);
// Maps facet-local points chi (D-1 coords each) to the element reference coordinates on facet f
// (Curvilinear::facetParam, src/geometry/Curvilinear.cpp:351-368).
Points facet_param(int D, int f, Points const& chi);
// Reference outward normals of the unit simplex facets (Curvilinear.cpp:128-164).
std::vector<std::array<double, 3>> reference_normals(int D);

}  // namespace tdg
