// Reference-element tables (see refelem.hpp).  Citations name the tandem source each routine
// restates; the code is written for this library's flat data layout.
#include "refelem.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <string>

namespace tdg {

// ---------------------------------------------------------------------------------------------
// small dense linear algebra
// ---------------------------------------------------------------------------------------------

Dense invert(Dense const& m) {
    if (m.rows != m.cols) throw std::invalid_argument("invert: matrix not square");
    int n = m.rows;
    Dense a = m;
    Dense inv(n, n);
    for (int i = 0; i < n; ++i) inv(i, i) = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        double best = std::fabs(a(c, c));
        for (int r = c + 1; r < n; ++r) {
            if (std::fabs(a(r, c)) > best) {
                best = std::fabs(a(r, c));
                piv = r;
            }
        }
        if (best == 0.0) throw std::runtime_error("invert: singular matrix");
        if (piv != c) {
            for (int j = 0; j < n; ++j) {
                std::swap(a(c, j), a(piv, j));
                std::swap(inv(c, j), inv(piv, j));
            }
        }
        double d = 1.0 / a(c, c);
        for (int j = 0; j < n; ++j) {
            a(c, j) *= d;
            inv(c, j) *= d;
        }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            double f = a(r, c);
            if (f == 0.0) continue;
            for (int j = 0; j < n; ++j) {
                a(r, j) -= f * a(c, j);
                inv(r, j) -= f * inv(c, j);
            }
        }
    }
    return inv;
}

void solve_in_place(Dense m, double* b) {
    int n = m.rows;
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    for (int c = 0; c < n; ++c) {
        int piv = c;
        double best = std::fabs(m(c, c));
        for (int r = c + 1; r < n; ++r) {
            if (std::fabs(m(r, c)) > best) {
                best = std::fabs(m(r, c));
                piv = r;
            }
        }
        if (best == 0.0) throw std::runtime_error("solve: singular matrix");
        if (piv != c) {
            for (int j = 0; j < n; ++j) std::swap(m(c, j), m(piv, j));
            std::swap(b[c], b[piv]);
        }
        for (int r = c + 1; r < n; ++r) {
            double f = m(r, c) / m(c, c);
            if (f == 0.0) continue;
            for (int j = c; j < n; ++j) m(r, j) -= f * m(c, j);
            b[r] -= f * b[c];
        }
    }
    for (int r = n - 1; r >= 0; --r) {
        double s = b[r];
        for (int j = r + 1; j < n; ++j) s -= m(r, j) * b[j];
        b[r] = s / m(r, r);
    }
}

// ---------------------------------------------------------------------------------------------
// multi-index enumeration
// ---------------------------------------------------------------------------------------------

std::vector<std::array<unsigned, 3>> graded_multi_indices(int D, unsigned N) {
    // A non-decreasing "marker" vector m_0 <= m_1 <= ... <= m_{D-1} walks through all
    // multi-indices; the index is the sequence of marker gaps read backwards.  Incrementing finds
    // the first marker that is smaller than its successor (or the last one), bumps it and resets
    // all markers before it.  This yields tandem's order: total degree first, then the first
    // component decreasing.
    std::vector<std::array<unsigned, 3>> out;
    std::array<unsigned, 3> m{0, 0, 0};
    for (;;) {
        if (m[D - 1] > N) break;
        std::array<unsigned, 3> j{0, 0, 0};
        j[D - 1] = m[0];
        for (int k = 1; k < D; ++k) j[D - 1 - k] = m[k] - m[k - 1];
        out.push_back(j);
        int d = 0;
        while (d < D - 1 && m[d] == m[d + 1]) ++d;
        ++m[d];
        for (int k = 0; k < d; ++k) m[k] = 0;
    }
    return out;
}

// ---------------------------------------------------------------------------------------------
// Jacobi and Dubiner polynomials
// ---------------------------------------------------------------------------------------------

double jacobi_p(unsigned n, unsigned a, unsigned b, double x) {
    if (n == 0) return 1.0;
    double p2 = 0.0, p1 = 1.0;
    double p = 0.5 * a - 0.5 * b + (1.0 + 0.5 * (a + b)) * x;
    double a2b2 = static_cast<double>(a * a) - static_cast<double>(b * b);
    for (unsigned m = 2; m <= n; ++m) {
        p2 = p1;
        p1 = p;
        double s = 2.0 * m + a + b;
        p = ((s - 1.0) * (a2b2 + s * (s - 2.0) * x) * p1 - 2.0 * (m + a - 1.0) * (m + b - 1.0) * s * p2) /
            (2.0 * m * (m + a + b) * (s - 2.0));
    }
    return p;
}

double jacobi_p_derivative(unsigned n, unsigned a, unsigned b, double x) {
    return n == 0 ? 0.0 : 0.5 * (n + a + b + 1.0) * jacobi_p(n - 1, a + 1, b + 1, x);
}

namespace {
// Recurrence coefficients of the homogenised Jacobi recurrence at step m.
struct SfCoeff {
    double c1, c2, c3, c4, c5;
};
SfCoeff sf_coeff(unsigned m, unsigned a, unsigned b) {
    double c0 = 2.0 * m + a + b;
    return {c0 - 1.0, static_cast<double>(a * a) - static_cast<double>(b * b), c0 * (c0 - 2.0),
            2.0 * (m + a - 1.0) * (m + b - 1.0) * c0, 2.0 * m * (m + a + b) * (c0 - 2.0)};
}
}  // namespace

double sf_jacobi_p(unsigned n, unsigned a, unsigned b, double x, double y) {
    if (n == 0) return 1.0;
    double p2 = 0.0, p1 = 1.0;
    double p = (0.5 * a - 0.5 * b) * y + (1.0 + 0.5 * (a + b)) * x;
    for (unsigned m = 2; m <= n; ++m) {
        p2 = p1;
        p1 = p;
        SfCoeff c = sf_coeff(m, a, b);
        p = (c.c1 * (c.c2 * y + c.c3 * x) * p1 - c.c4 * y * y * p2) / c.c5;
    }
    return p;
}

std::array<double, 3> sf_jacobi_p_and_derivatives(unsigned n, unsigned a, unsigned b, double x,
                                                  double y) {
    if (n == 0) return {1.0, 0.0, 0.0};
    double p2 = 0.0, p1 = 1.0, dx2 = 0.0, dx1 = 0.0, dy2 = 0.0, dy1 = 0.0;
    double p = sf_jacobi_p(1, a, b, x, y);
    double dx = 1.0 + 0.5 * (a + b);
    double dy = 0.5 * (static_cast<double>(a) - static_cast<double>(b));
    for (unsigned m = 2; m <= n; ++m) {
        p2 = p1;
        p1 = p;
        dx2 = dx1;
        dx1 = dx;
        dy2 = dy1;
        dy1 = dy;
        SfCoeff c = sf_coeff(m, a, b);
        double lin = c.c2 * y + c.c3 * x;
        p = (c.c1 * lin * p1 - c.c4 * y * y * p2) / c.c5;
        dx = (c.c1 * (c.c3 * p1 + lin * dx1) - c.c4 * y * y * dx2) / c.c5;
        dy = (c.c1 * (c.c2 * p1 + lin * dy1) - c.c4 * (2.0 * y * p2 + y * y * dy2)) / c.c5;
    }
    return {p, dx, dy};
}

double dubiner(int D, std::array<unsigned, 3> const& j, double const* xi) {
    if (D == 1) return jacobi_p(j[0], 0, 0, 2.0 * xi[0] - 1.0);
    if (D == 2) {
        double r = 2.0 * xi[0] - 1.0 + xi[1];
        double s = 2.0 * xi[1] - 1.0;
        double th = 1.0 - xi[1];
        return sf_jacobi_p(j[0], 0, 0, r, th) * sf_jacobi_p(j[1], 2 * j[0] + 1, 0, s, 1.0);
    }
    double r = 2.0 * xi[0] - 1.0 + xi[1] + xi[2];
    double s = 2.0 * xi[1] - 1.0 + xi[2];
    double t = 2.0 * xi[2] - 1.0;
    double st = 1.0 - xi[1] - xi[2];
    double th = 1.0 - xi[2];
    return sf_jacobi_p(j[0], 0, 0, r, st) * sf_jacobi_p(j[1], 2 * j[0] + 1, 0, s, th) *
           sf_jacobi_p(j[2], 2 * j[0] + 2 * j[1] + 2, 0, t, 1.0);
}

std::array<double, 3> grad_dubiner(int D, std::array<unsigned, 3> const& j, double const* xi) {
    if (D == 1) {
        // tandem returns dP/dx at x = 2 xi - 1 here (src/basis/Functions.h:147-150); kept as is.
        return {jacobi_p_derivative(j[0], 0, 0, 2.0 * xi[0] - 1.0), 0.0, 0.0};
    }
    if (D == 2) {
        double r = 2.0 * xi[0] - 1.0 + xi[1];
        double s = 2.0 * xi[1] - 1.0;
        double th = 1.0 - xi[1];
        auto a = sf_jacobi_p_and_derivatives(j[0], 0, 0, r, th);
        auto b = sf_jacobi_p_and_derivatives(j[1], 2 * j[0] + 1, 0, s, 1.0);
        // d/dxi0: dr = 2;  d/dxi1: dr = 1, dth = -1, ds = 2
        double g0 = (a[1] * 2.0) * b[0];
        double g1 = (a[1] * 1.0 - a[2]) * b[0] + a[0] * b[1] * 2.0;
        return {g0, g1, 0.0};
    }
    double r = 2.0 * xi[0] - 1.0 + xi[1] + xi[2];
    double s = 2.0 * xi[1] - 1.0 + xi[2];
    double t = 2.0 * xi[2] - 1.0;
    double st = 1.0 - xi[1] - xi[2];
    double th = 1.0 - xi[2];
    auto a = sf_jacobi_p_and_derivatives(j[0], 0, 0, r, st);
    auto b = sf_jacobi_p_and_derivatives(j[1], 2 * j[0] + 1, 0, s, th);
    auto c = sf_jacobi_p_and_derivatives(j[2], 2 * j[0] + 2 * j[1] + 2, 0, t, 1.0);
    auto d = [&](double dr, double dst, double ds, double dth, double dt) {
        return (a[1] * dr + a[2] * dst) * b[0] * c[0] + a[0] * (b[1] * ds + b[2] * dth) * c[0] +
               a[0] * b[0] * (c[1] * dt);
    };
    return {d(2.0, 0.0, 0.0, 0.0, 0.0), d(1.0, -1.0, 2.0, 0.0, 0.0), d(1.0, -1.0, 1.0, -1.0, 2.0)};
}

// ---------------------------------------------------------------------------------------------
// quadrature
// ---------------------------------------------------------------------------------------------

IntervalRule gauss_jacobi(unsigned n, unsigned a, unsigned b) {
    constexpr double tol = 10.0 * std::numeric_limits<double>::epsilon();
    constexpr unsigned max_it = 100;
    auto prod = [](std::uint64_t from, std::uint64_t to) {
        std::uint64_t p = 1;
        for (; from <= to; ++from) p *= from;
        return static_cast<double>(p);
    };
    IntervalRule rule;
    rule.x.resize(n);
    rule.w.resize(n);
    // Weight formula for the Gauss-Jacobi rule expressed through P_{n+1} and P_n'.
    double wf = -(2.0 * n + a + b + 2) * prod(n + 1, n + b) * static_cast<double>(1u << (a + b)) /
                ((n + a + b + 1.0) * prod(n + a + 1, n + a + b) * (n + 1));
    for (unsigned i = 1; i <= n; ++i) {
        double x = std::cos(M_PI * (0.5 * a + i - 0.25) / (0.5 * (1.0 + a + b) + n));
        double p = 0.0, dp = 1.0;
        unsigned it = 0;
        do {
            x -= p / dp;
            p = jacobi_p(n, a, b, x);
            dp = jacobi_p_derivative(n, a, b, x);
        } while (std::fabs(p) > tol && ++it < max_it);
        rule.x[i - 1] = x;
        rule.w[i - 1] = wf / (jacobi_p(n + 1, a, b, x) * dp);
    }
    return rule;
}

std::vector<double> lgl_points(unsigned n) {
    if (n < 2) throw std::invalid_argument("lgl_points: n >= 2 required");
    auto gj = gauss_jacobi(n - 2, 1, 1);
    std::vector<double> out;
    out.push_back(-1.0);
    for (auto it = gj.x.rbegin(); it != gj.x.rend(); ++it) out.push_back(*it);
    out.push_back(1.0);
    return out;
}

namespace {
IntervalRule unit_interval(IntervalRule r) {
    for (auto& x : r.x) x = 0.5 * x + 0.5;
    for (auto& w : r.w) w *= 0.5;
    return r;
}
}  // namespace

SimplexRule conical_product_rule(int D, unsigned min_order) {
    unsigned n = 1 + min_order / 2;
    SimplexRule rule;
    rule.dim = D;
    rule.order = static_cast<int>(2 * n - 1);
    auto g0 = unit_interval(gauss_jacobi(n, 0, 0));
    if (D == 1) {
        rule.x = g0.x;
        rule.w = g0.w;
        return rule;
    }
    auto g1 = unit_interval(gauss_jacobi(n, 1, 0));
    if (D == 2) {
        for (unsigned i = 0; i < n; ++i) {
            for (unsigned j = 0; j < n; ++j) {
                rule.x.push_back(g1.x[i]);
                rule.x.push_back(g0.x[j] * (1.0 - g1.x[i]));
                rule.w.push_back(0.5 * g1.w[i] * g0.w[j]);
            }
        }
        return rule;
    }
    auto g2 = unit_interval(gauss_jacobi(n, 2, 0));
    for (unsigned i = 0; i < n; ++i) {
        for (unsigned j = 0; j < n; ++j) {
            for (unsigned k = 0; k < n; ++k) {
                rule.x.push_back(g2.x[i]);
                rule.x.push_back(g1.x[j] * (1.0 - g2.x[i]));
                rule.x.push_back(g0.x[k] * (1.0 - g1.x[j]) * (1.0 - g2.x[i]));
                rule.w.push_back(0.125 * g2.w[i] * g1.w[j] * g0.w[k]);
            }
        }
    }
    return rule;
}

// ---------------------------------------------------------------------------------------------
// nodes
// ---------------------------------------------------------------------------------------------

namespace {

// Optimised warp & blend blending parameters alpha(N), N = 1..15, from Hesthaven & Warburton
// (Nodal Discontinuous Galerkin Methods, 2008); tandem tabulates the same published values
// (src/basis/WarpAndBlend.cpp:25-37) and uses 5/3 beyond its table.
double wb_alpha(int D, unsigned N) {
    static const double a2[] = {0.0000, 0.0000, 1.4152, 0.1001, 0.2751, 0.9800, 1.0999, 1.2832,
                                1.3648, 1.4773, 1.4959, 1.5743, 1.5770, 1.6223, 1.6258};
    static const double a3[] = {0.0,    0.0,    0.0,     0.1002, 1.1332, 1.5608, 1.3413, 1.2577,
                                1.1603, 1.10153, 0.6080, 0.4523, 0.8856, 0.8717, 0.9655};
    if (N < 1 || N > 15) throw std::invalid_argument("warp & blend: degree must be in [1, 15]");
    return D == 2 ? a2[N - 1] : a3[N - 1];
}

using Vec3 = std::array<double, 3>;

std::array<Vec3, 3> equilateral_triangle() {
    return {Vec3{-1.0, -1.0 / std::sqrt(3.0), 0.0}, Vec3{1.0, -1.0 / std::sqrt(3.0), 0.0},
            Vec3{0.0, 2.0 / std::sqrt(3.0), 0.0}};
}
std::array<Vec3, 4> equilateral_tet() {
    return {Vec3{-1.0, -1.0 / std::sqrt(3.0), -1.0 / std::sqrt(6.0)},
            Vec3{1.0, -1.0 / std::sqrt(3.0), -1.0 / std::sqrt(6.0)},
            Vec3{0.0, 2.0 / std::sqrt(3.0), -1.0 / std::sqrt(6.0)},
            Vec3{0.0, 0.0, 3.0 / std::sqrt(6.0)}};
}

// 1D warp function: interpolant of (LGL - equidistant) node displacement, evaluated at r and
// divided by the edge bubble 1 - r^2 (src/basis/WarpAndBlend.cpp:164-205).
struct Warp {
    unsigned N;
    std::vector<double> diff;
    Dense VTinv;  // inverse of V^T with V(i, j) = P_j(eq_i)
    explicit Warp(unsigned n) : N(n), diff(n + 1) {
        std::vector<double> eq(n + 1);
        for (unsigned i = 0; i <= n; ++i) eq[i] = 2.0 * i / static_cast<double>(n) - 1.0;
        Dense VT(n + 1, n + 1);
        for (unsigned i = 0; i <= n; ++i)
            for (unsigned j = 0; j <= n; ++j) VT(j, i) = jacobi_p(j, 0, 0, eq[i]);
        VTinv = invert(VT);
        auto gl = lgl_points(n + 1);
        for (unsigned i = 0; i <= n; ++i) diff[i] = gl[i] - eq[i];
    }
    double operator()(double r) const {
        // Lagrange weights L = V^-T phi(r), warp = L . diff
        std::vector<double> phi(N + 1);
        for (unsigned i = 0; i <= N; ++i) phi[i] = jacobi_p(i, 0, 0, r);
        double w = 0.0;
        for (unsigned i = 0; i <= N; ++i) {
            double li = 0.0;
            for (unsigned k = 0; k <= N; ++k) li += VTinv(i, k) * phi[k];
            w += li * diff[i];
        }
        if (std::fabs(r) < 1.0 - std::numeric_limits<double>::epsilon()) w /= 1.0 - r * r;
        return w;
    }
};

// Warp & blend displacement on an equilateral triangle for barycentric rows L (n x 3); returns
// n x 2 displacements (src/basis/WarpAndBlend.cpp:207-231).
std::vector<std::array<double, 2>> wb_triangle(unsigned N, double alpha,
                                               std::vector<Vec3> const& L) {
    auto eqv = equilateral_triangle();
    Warp warp(N);
    std::vector<std::array<double, 2>> out(L.size(), {0.0, 0.0});
    auto fv = facet_vertices(2);
    for (auto const& f : fv) {
        int v0 = f[0], v1 = f[1];
        int mv = 3 - v0 - v1;
        double tx = eqv[v1][0] - eqv[v0][0], ty = eqv[v1][1] - eqv[v0][1];
        double tn = std::sqrt(tx * tx + ty * ty);
        tx /= tn;
        ty /= tn;
        for (std::size_t i = 0; i < L.size(); ++i) {
            double w = warp(L[i][v1] - L[i][v0]);
            double blend = 4.0 * L[i][v0] * L[i][v1];
            blend *= 1.0 + alpha * alpha * L[i][mv] * L[i][mv];
            out[i][0] += w * blend * tx;
            out[i][1] += w * blend * ty;
        }
    }
    return out;
}

// Maps a point of the simplex spanned by `verts` to unit-simplex coordinates.
template <int D>
std::array<double, D> to_reference(std::array<Vec3, D + 1> const& verts, Vec3 const& x) {
    Dense A(D, D);
    std::array<double, D> rhs{};
    for (int i = 0; i < D; ++i) {
        for (int j = 0; j < D; ++j) A(i, j) = verts[j + 1][i] - verts[0][i];
        rhs[i] = x[i] - verts[0][i];
    }
    solve_in_place(A, rhs.data());
    return rhs;
}

}  // namespace

Points warp_blend_nodes(int D, unsigned N) {
    Points out;
    if (D == 1) {
        if (N == 0) return {0.5};
        auto gl = lgl_points(N + 1);
        for (double g : gl) out.push_back(0.5 * g + 0.5);
        return out;
    }
    auto idx = graded_multi_indices(D, N);
    std::size_t n = idx.size();
    if (N == 0) {
        for (int d = 0; d < D; ++d) out.push_back(1.0 / (D + 1));
        return out;
    }
    double alpha = wb_alpha(D, N);
    if (D == 2) {
        auto eqv = equilateral_triangle();
        std::vector<Vec3> L(n);
        for (std::size_t i = 0; i < n; ++i) {
            L[i][2] = idx[i][1] / static_cast<double>(N);
            L[i][1] = idx[i][0] / static_cast<double>(N);
            L[i][0] = 1.0 - L[i][1] - L[i][2];
        }
        auto wb = wb_triangle(N, alpha, L);
        std::array<Vec3, 3> verts = eqv;
        for (std::size_t i = 0; i < n; ++i) {
            Vec3 x{0.0, 0.0, 0.0};
            for (int v = 0; v < 3; ++v) {
                x[0] += L[i][v] * eqv[v][0];
                x[1] += L[i][v] * eqv[v][1];
            }
            x[0] += wb[i][0];
            x[1] += wb[i][1];
            auto xi = to_reference<2>(verts, x);
            out.push_back(xi[0]);
            out.push_back(xi[1]);
        }
        return out;
    }
    // D == 3
    auto eqv = equilateral_tet();
    std::vector<std::array<double, 4>> L(n);
    for (std::size_t i = 0; i < n; ++i) {
        L[i][3] = idx[i][2] / static_cast<double>(N);
        L[i][2] = idx[i][1] / static_cast<double>(N);
        L[i][1] = idx[i][0] / static_cast<double>(N);
        L[i][0] = 1.0 - L[i][1] - L[i][2] - L[i][3];
    }
    std::vector<Vec3> res(n, Vec3{0.0, 0.0, 0.0});
    for (auto const& f : facet_vertices(3)) {
        int mv = 6 - f[0] - f[1] - f[2];
        Vec3 t0, t1;
        double n0 = 0.0, n1 = 0.0;
        for (int d = 0; d < 3; ++d) {
            t0[d] = eqv[f[1]][d] - eqv[f[0]][d];
            t1[d] = eqv[f[2]][d] - 0.5 * (eqv[f[1]][d] + eqv[f[0]][d]);
            n0 += t0[d] * t0[d];
            n1 += t1[d] * t1[d];
        }
        for (int d = 0; d < 3; ++d) {
            t0[d] /= std::sqrt(n0);
            t1[d] /= std::sqrt(n1);
        }
        std::vector<Vec3> Lf(n);
        for (std::size_t i = 0; i < n; ++i) Lf[i] = {L[i][f[0]], L[i][f[1]], L[i][f[2]]};
        auto w2 = wb_triangle(N, alpha, Lf);
        for (std::size_t i = 0; i < n; ++i) {
            double lm = L[i][mv];
            double blend = Lf[i][0] * Lf[i][1] * Lf[i][2];
            double denom = (Lf[i][0] + 0.5 * lm) * (Lf[i][1] + 0.5 * lm) * (Lf[i][2] + 0.5 * lm);
            double factor = 1.0 + alpha * alpha * lm * lm;
            double mask;
            if (std::fabs(denom) < std::numeric_limits<double>::epsilon()) {
                blend = 1.0;
                mask = 0.0;
            } else {
                blend = factor * blend / denom;
                mask = 1.0;
            }
            for (int d = 0; d < 3; ++d) {
                double w = w2[i][0] * t0[d] + w2[i][1] * t1[d];
                res[i][d] = mask * res[i][d] + blend * w;
            }
        }
    }
    for (std::size_t i = 0; i < n; ++i) {
        Vec3 x = res[i];
        for (int v = 0; v < 4; ++v)
            for (int d = 0; d < 3; ++d) x[d] += L[i][v] * eqv[v][d];
        auto xi = to_reference<3>(eqv, x);
        out.push_back(xi[0]);
        out.push_back(xi[1]);
        out.push_back(xi[2]);
    }
    return out;
}

namespace {
template <int DD>
void shrink(double factor, std::array<Vec3, DD + 1>& v) {
    std::array<Vec3, DD + 1> r{};
    for (int i = 0; i <= DD; ++i)
        for (int j = 0; j <= DD; ++j) {
            double l = (i == j) ? 1.0 - DD * factor : factor;
            for (int d = 0; d < 3; ++d) r[i][d] += l * v[j][d];
        }
    v = r;
}
void edge_nodes(int n, Vec3 const& a, Vec3 const& b, std::vector<Vec3>& out) {
    double h = 1.0 / (n + 1);
    for (int k = 1; k <= n; ++k) {
        double l = k * h;
        out.push_back({(1 - l) * a[0] + l * b[0], (1 - l) * a[1] + l * b[1], (1 - l) * a[2] + l * b[2]});
    }
}
void tri_nodes(int n, std::array<Vec3, 3> v, std::vector<Vec3>& out) {
    while (n >= 0) {
        out.push_back(v[0]);
        if (n > 0) {
            out.push_back(v[1]);
            out.push_back(v[2]);
            edge_nodes(n - 1, v[0], v[1], out);
            edge_nodes(n - 1, v[1], v[2], out);
            edge_nodes(n - 1, v[2], v[0], out);
            shrink<2>(1.0 / n, v);
        }
        n -= 3;
    }
}
}  // namespace

Points equidistant_nodes(int D, unsigned N) {
    // VTK numbering: corner nodes, then edge-interior nodes edge by edge, then face and interior
    // nodes recursively (src/basis/Equidistant.cpp, src/basis/NumberingConvention.h).
    std::vector<Vec3> out;
    if (D == 2) {
        tri_nodes(static_cast<int>(N), {Vec3{0, 0, 0}, Vec3{1, 0, 0}, Vec3{0, 1, 0}}, out);
    } else if (D == 3) {
        static const int edges[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
        static const int faces[4][3] = {{0, 1, 3}, {2, 3, 1}, {0, 3, 2}, {0, 2, 1}};
        std::array<Vec3, 4> v{Vec3{0, 0, 0}, Vec3{1, 0, 0}, Vec3{0, 1, 0}, Vec3{0, 0, 1}};
        int n = static_cast<int>(N);
        while (n >= 0) {
            out.push_back(v[0]);
            if (n > 0) {
                for (int k = 1; k < 4; ++k) out.push_back(v[k]);
                for (auto const& e : edges) edge_nodes(n - 1, v[e[0]], v[e[1]], out);
                double sf = 1.0 / n;
                if (n >= 3) {
                    for (auto const& f : faces) {
                        std::array<Vec3, 3> fv{v[f[0]], v[f[1]], v[f[2]]};
                        shrink<2>(sf, fv);
                        tri_nodes(n - 3, fv, out);
                    }
                }
                shrink<3>(sf, v);
            }
            n -= 4;
        }
    } else {
        throw std::invalid_argument("equidistant_nodes: D must be 2 or 3");
    }
    Points p;
    for (auto const& x : out)
        for (int d = 0; d < D; ++d) p.push_back(x[d]);
    return p;
}

Dense vandermonde(int D, unsigned N, Points const& nodes) {
    auto idx = graded_multi_indices(D, N);
    int n = static_cast<int>(nodes.size() / D);
    Dense V(n, static_cast<int>(idx.size()));
    for (int i = 0; i < n; ++i)
        for (std::size_t j = 0; j < idx.size(); ++j)
            V(i, static_cast<int>(j)) = dubiner(D, idx[j], &nodes[static_cast<std::size_t>(i) * D]);
    return V;
}

// ---------------------------------------------------------------------------------------------
// reference spaces
// ---------------------------------------------------------------------------------------------

RefSpace RefSpace::modal(int D, unsigned N) {
    RefSpace s;
    s.D_ = D;
    s.N_ = static_cast<int>(N);
    s.idx_ = graded_multi_indices(D, N);
    s.nbf_ = static_cast<int>(s.idx_.size());
    return s;
}

RefSpace RefSpace::nodal(int D, unsigned N, Points nodes) {
    RefSpace s = modal(D, N);
    s.nodal_ = true;
    s.nodes_ = std::move(nodes);
    if (static_cast<int>(s.nodes_.size()) != s.nbf_ * D)
        throw std::invalid_argument("nodal space: node count does not match degree");
    s.Vinv_ = invert(vandermonde(D, N, s.nodes_));
    return s;
}

Dense RefSpace::eval(Points const& pts) const {
    int np = static_cast<int>(pts.size() / D_);
    Dense modalE(nbf_, np);
    for (int q = 0; q < np; ++q)
        for (int k = 0; k < nbf_; ++k)
            modalE(k, q) = dubiner(D_, idx_[k], &pts[static_cast<std::size_t>(q) * D_]);
    if (!nodal_) return modalE;
    // nodal basis: phi_i = sum_j Vinv(j, i) psi_j
    Dense E(nbf_, np);
    for (int i = 0; i < nbf_; ++i)
        for (int q = 0; q < np; ++q) {
            double s = 0.0;
            for (int j = 0; j < nbf_; ++j) s += Vinv_(j, i) * modalE(j, q);
            E(i, q) = s;
        }
    return E;
}

std::vector<double> RefSpace::grad(Points const& pts) const {
    int np = static_cast<int>(pts.size() / D_);
    std::vector<double> g(static_cast<std::size_t>(nbf_) * D_ * np);
    for (int q = 0; q < np; ++q)
        for (int k = 0; k < nbf_; ++k) {
            auto d = grad_dubiner(D_, idx_[k], &pts[static_cast<std::size_t>(q) * D_]);
            for (int e = 0; e < D_; ++e) g[(static_cast<std::size_t>(k) * D_ + e) * np + q] = d[e];
        }
    if (!nodal_) return g;
    std::vector<double> out(g.size(), 0.0);
    for (int i = 0; i < nbf_; ++i)
        for (int j = 0; j < nbf_; ++j) {
            double v = Vinv_(j, i);
            if (v == 0.0) continue;
            for (int e = 0; e < D_; ++e)
                for (int q = 0; q < np; ++q)
                    out[(static_cast<std::size_t>(i) * D_ + e) * np + q] +=
                        v * g[(static_cast<std::size_t>(j) * D_ + e) * np + q];
        }
    return out;
}

Dense RefSpace::mass_matrix() const {
    auto rule = conical_product_rule(D_, 2 * N_);
    RefSpace m = modal(D_, N_);
    Dense E = m.eval(rule.x);
    Dense M(nbf_, nbf_);
    for (int i = 0; i < nbf_; ++i) {
        double s = 0.0;
        for (int q = 0; q < rule.size(); ++q) s += rule.w[q] * E(i, q) * E(i, q);
        M(i, i) = s;  // Dubiner polynomials are orthogonal
    }
    if (!nodal_) return M;
    Dense R(nbf_, nbf_);
    for (int i = 0; i < nbf_; ++i)
        for (int j = 0; j < nbf_; ++j) {
            double s = 0.0;
            for (int k = 0; k < nbf_; ++k) s += Vinv_(k, i) * M(k, k) * Vinv_(k, j);
            R(i, j) = s;
        }
    return R;
}

// ---------------------------------------------------------------------------------------------
// reference simplex facets
// ---------------------------------------------------------------------------------------------

std::vector<std::array<int, 3>> facet_vertices(int D) {
    // D-subsets of {0..D} in lexicographic order
    if (D == 1) return {{0, 0, 0}, {1, 0, 0}};
    if (D == 2) return {{0, 1, 0}, {0, 2, 0}, {1, 2, 0}};
    return {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
}

namespace {
Vec3 ref_vertex(int D, int v) {
    Vec3 x{0.0, 0.0, 0.0};
    if (v > 0) x[v - 1] = 1.0;
    (void)D;
    return x;
}
}  // namespace

Points facet_param(int D, int f, Points const& chi) {
    auto fv = facet_vertices(D)[f];
    int dd = D - 1;
    int n = dd == 0 ? 1 : static_cast<int>(chi.size() / dd);
    Points out;
    for (int p = 0; p < n; ++p) {
        double s = 0.0;
        for (int d = 0; d < dd; ++d) s += chi[static_cast<std::size_t>(p) * dd + d];
        Vec3 v0 = ref_vertex(D, fv[0]);
        Vec3 xi{(1.0 - s) * v0[0], (1.0 - s) * v0[1], (1.0 - s) * v0[2]};
        for (int d = 0; d < dd; ++d) {
            Vec3 vd = ref_vertex(D, fv[d + 1]);
            double c = chi[static_cast<std::size_t>(p) * dd + d];
            for (int k = 0; k < 3; ++k) xi[k] += c * vd[k];
        }
        for (int k = 0; k < D; ++k) out.push_back(xi[k]);
    }
    return out;
}

std::vector<std::array<double, 3>> reference_normals(int D) {
    std::vector<std::array<double, 3>> out;
    for (auto const& f : facet_vertices(D)) {
        Vec3 n{0.0, 0.0, 0.0};
        Vec3 a = ref_vertex(D, f[0]), b = ref_vertex(D, f[1]);
        if (D == 2) {
            n = {-(b[1] - a[1]), b[0] - a[0], 0.0};
        } else {
            Vec3 c = ref_vertex(D, f[2]);
            Vec3 e1{b[0] - a[0], b[1] - a[1], b[2] - a[2]};
            Vec3 e2{c[0] - a[0], c[1] - a[1], c[2] - a[2]};
            n = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                 e1[0] * e2[1] - e1[1] * e2[0]};
        }
        int mv = (D == 2) ? 3 - f[0] - f[1] : 6 - f[0] - f[1] - f[2];
        Vec3 m = ref_vertex(D, mv);
        double dot = 0.0;
        for (int k = 0; k < D; ++k) dot += n[k] * (m[k] - a[k]);
        if (dot > 0) {
            for (auto& x : n) x = -x;
        }
        out.push_back(n);
    }
    return out;
}

}  // namespace tdg
