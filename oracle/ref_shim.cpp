// ORACLE -- test infrastructure only.  C entry points over tandem's own quadrature and basis
// sources, compiled in place from the reference tree (see oracle/build.py) into
// oracle/_ref/libtandem_ref.so.  Used to pin the restatements (quadrature rules, Dubiner
// polynomials, Gauss-Jacobi) and to generate the committed golden fixtures.
#include "basis/Functions.h"
#include "quadrules/AutoRule.h"
#include "quadrules/GaussJacobi.h"
#include "quadrules/TensorProductRule.h"

#include <array>
#include <cstring>

using namespace tndm;

extern "C" {

// tandem's simplexQuadratureRule<D>(order) (src/quadrules/AutoRule.h:41-50); returns its size and
// fills points [n][dim] / weights [n] when non-null.
int ref_simplex_rule(int dim, int order, double* pts, double* wts) {
    auto copy = [&](auto const& rule, int D) {
        auto n = static_cast<int>(rule.size());
        if (pts)
            for (int i = 0; i < n; ++i)
                for (int d = 0; d < D; ++d) pts[i * D + d] = rule.points()[i][d];
        if (wts)
            for (int i = 0; i < n; ++i) wts[i] = rule.weights()[i];
        return n;
    };
    if (dim == 1) return copy(simplexQuadratureRule<1u>(order), 1);
    if (dim == 2) return copy(simplexQuadratureRule<2u>(order), 2);
    if (dim == 3) return copy(simplexQuadratureRule<3u>(order), 3);
    return -1;
}

int ref_conical_rule(int dim, int order, double* pts, double* wts) {
    auto copy = [&](auto rule, int D) {
        auto n = static_cast<int>(rule.size());
        if (pts)
            for (int i = 0; i < n; ++i)
                for (int d = 0; d < D; ++d) pts[i * D + d] = rule.points()[i][d];
        if (wts)
            for (int i = 0; i < n; ++i) wts[i] = rule.weights()[i];
        return n;
    };
    if (dim == 1) return copy(TensorProductRule<1u>::get(order), 1);
    if (dim == 2) return copy(TensorProductRule<2u>::get(order), 2);
    if (dim == 3) return copy(TensorProductRule<3u>::get(order), 3);
    return -1;
}

int ref_gauss_jacobi(int n, int a, int b, double* x, double* w) {
    auto r = GaussJacobi(n, a, b);
    for (int i = 0; i < n; ++i) {
        x[i] = r.points()[i];
        w[i] = r.weights()[i];
    }
    return n;
}

double ref_jacobi(int n, int a, int b, double x) { return JacobiP(n, a, b, x); }

double ref_dubiner(int dim, const unsigned* j, const double* xi) {
    if (dim == 2) return DubinerP<2>({j[0], j[1]}, {xi[0], xi[1]});
    return DubinerP<3>({j[0], j[1], j[2]}, {xi[0], xi[1], xi[2]});
}

void ref_grad_dubiner(int dim, const unsigned* j, const double* xi, double* out) {
    if (dim == 2) {
        auto g = gradDubinerP<2>({j[0], j[1]}, {xi[0], xi[1]});
        out[0] = g[0];
        out[1] = g[1];
        return;
    }
    auto g = gradDubinerP<3>({j[0], j[1], j[2]}, {xi[0], xi[1], xi[2]});
    out[0] = g[0];
    out[1] = g[1];
    out[2] = g[2];
}

}  // extern "C"
