// Host-side operator set-up (see setup.hpp).  Restates, for this library's flat layout:
//  - Curvilinear::jacobian / jacobianInv / absDetJ / normal / map
//    (src/geometry/Curvilinear.cpp:174-274),
//  - DGCurvilinearCommon::prepare_volume / prepare_bndskl (src/form/DGCurvilinearCommon.cpp:41-102),
//  - Poisson::prepare_* and Elasticity::prepare_* (app/localoperator/Poisson.cpp:133-223,
//    app/localoperator/Elasticity.cpp:104-292),
//  - the facet-side tables of DGOperatorTopo (src/form/DGOperatorTopo.cpp:46-85),
//  - Poisson/Elasticity rhs_* with the interior-penalty lift (Poisson.cpp:387-549,
//    Elasticity.cpp:521-696).
#include "setup.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>

namespace tdg {

namespace {

constexpr int kPoisson = 0;

// Inverse and determinant of a D x D matrix stored row-major a[i * D + j].
double inv_det(int D, double const* a, double* inv) {
    if (D == 2) {
        double det = a[0] * a[3] - a[1] * a[2];
        double id = 1.0 / det;
        inv[0] = a[3] * id;
        inv[1] = -a[1] * id;
        inv[2] = -a[2] * id;
        inv[3] = a[0] * id;
        return det;
    }
    double c00 = a[4] * a[8] - a[5] * a[7];
    double c01 = a[5] * a[6] - a[3] * a[8];
    double c02 = a[3] * a[7] - a[4] * a[6];
    double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    double id = 1.0 / det;
    inv[0] = c00 * id;
    inv[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    inv[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    inv[3] = c01 * id;
    inv[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    inv[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    inv[6] = c02 * id;
    inv[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    inv[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    return det;
}

// Trace inverse inequality constant c_N = (N + 1)(N + D) / D (Warburton & Hesthaven 2003;
// src/form/InverseInequality.h:27-29).
double trace_constant(int D, int N) { return (N + 1.0) * (N + D) / static_cast<double>(D); }

}  // namespace

void HostOperator::build(int D_, int N_, int geoN_, int kind_, int64_t E_, int64_t F_,
                         double const* geo, int64_t const* facet_up, int32_t const* facet_loc,
                         int32_t const* facet_bc, int nvol, double const* vx, double const* vw,
                         int nfct, double const* fx, double const* fw) {
    if (D_ != 2 && D_ != 3) throw std::invalid_argument("dim must be 2 or 3");
    if (N_ < 1 || N_ > 8) throw std::invalid_argument("degree must be in [1, 8]");
    if (geoN_ < 1 || geoN_ > 8) throw std::invalid_argument("geo_degree must be in [1, 8]");
    if (kind_ != 0 && kind_ != 1) throw std::invalid_argument("kind must be POISSON or ELASTICITY");
    if (E_ <= 0 || F_ <= 0 || nvol <= 0 || nfct <= 0)
        throw std::invalid_argument("empty mesh or quadrature");
    D = D_;
    N = N_;
    geoN = geoN_;
    kind = kind_;
    E = E_;
    F = F_;
    nfaces = D + 1;
    Q = (kind == kPoisson) ? 1 : D;
    Nbf = num_basis(D, N);
    bs = Nbf * Q;
    Nq = nvol;
    nq = nfct;
    Ngeo = num_basis(D, geoN);
    ncoef = (kind == kPoisson) ? 1 : 2;

    vol_x.assign(vx, vx + static_cast<std::size_t>(Nq) * D);
    W.assign(vw, vw + Nq);
    fct_x.assign(fx, fx + static_cast<std::size_t>(nq) * (D - 1));
    w.assign(fw, fw + nq);

    // spaces: Poisson uses the modal Dubiner space (Poisson.h:131), Elasticity the nodal warp &
    // blend space (Elasticity.cpp:27-33); material and geometry are nodal warp & blend.
    auto wb = warp_blend_nodes(D, N);
    space = (kind == kPoisson) ? RefSpace::modal(D, N) : RefSpace::nodal(D, N, wb);
    mat_space = RefSpace::nodal(D, N, wb);
    geo_space = RefSpace::nodal(D, geoN, warp_blend_nodes(D, geoN));

    E_Q = space.eval(vol_x);
    Dxi_Q = space.grad(vol_x);
    matE_Q = mat_space.eval(vol_x);
    E_qf.clear();
    Dxi_qf.clear();
    matE_qf.clear();
    std::vector<Points> fpts(nfaces);
    for (int f = 0; f < nfaces; ++f) {
        fpts[f] = facet_param(D, f, fct_x);
        E_qf.push_back(space.eval(fpts[f]));
        Dxi_qf.push_back(space.grad(fpts[f]));
        matE_qf.push_back(mat_space.eval(fpts[f]));
    }

    // topology
    up.assign(facet_up, facet_up + 2 * F);
    loc.assign(facet_loc, facet_loc + 2 * F);
    bc.assign(facet_bc, facet_bc + F);
    sides.assign(static_cast<std::size_t>(E) * nfaces, Side{-1, -1, -1, -1, 0});
    for (int64_t f = 0; f < F; ++f) {
        for (int s = 0; s < 2; ++s) {
            int64_t el = up[2 * f + s];
            int l = loc[2 * f + s];
            if (el < 0 || el >= E || l < 0 || l >= nfaces)
                throw std::invalid_argument("facet " + std::to_string(f) + ": bad element/face");
            Side& sd = sides[static_cast<std::size_t>(el) * nfaces + l];
            sd.fct = static_cast<int32_t>(f);
            sd.side = s;
            sd.nb = static_cast<int32_t>(up[2 * f + 1 - s]);
            sd.nb_local = loc[2 * f + 1 - s];
            sd.bc = bc[f];
        }
    }
    for (auto const& sd : sides)
        if (sd.fct < 0) throw std::invalid_argument("an element face has no facet");

    // geometry at volume points
    geo_nodes.assign(geo, geo + static_cast<std::size_t>(E) * Ngeo * D);
    Dense geoE_Q = geo_space.eval(vol_x);
    auto geoD_Q = geo_space.grad(vol_x);
    std::vector<Dense> geoE_q;
    std::vector<std::vector<double>> geoD_q;
    for (int f = 0; f < nfaces; ++f) {
        geoE_q.push_back(geo_space.eval(fpts[f]));
        geoD_q.push_back(geo_space.grad(fpts[f]));
    }
    int DD = D * D;
    vG.assign(static_cast<std::size_t>(E) * DD * Nq, 0.0);
    vAbsDetJ.assign(static_cast<std::size_t>(E) * Nq, 0.0);
    vCoords.assign(static_cast<std::size_t>(E) * Nq * D, 0.0);
    volume.assign(E, 0.0);

    // J(i, e) = sum_n x_i(n) dphi_n/dxi_e at point q (Curvilinear::jacobian)
    auto jac = [&](int64_t el, std::vector<double> const& gd, int np, int q, double* J) {
        double const* X = &geo_nodes[static_cast<std::size_t>(el) * Ngeo * D];
        for (int i = 0; i < D; ++i)
            for (int e = 0; e < D; ++e) {
                double s = 0.0;
                for (int n = 0; n < Ngeo; ++n)
                    s += X[n * D + i] * gd[(static_cast<std::size_t>(n) * D + e) * np + q];
                J[i * D + e] = s;
            }
    };
    auto map = [&](int64_t el, Dense const& ge, int q, double* x) {
        double const* X = &geo_nodes[static_cast<std::size_t>(el) * Ngeo * D];
        for (int i = 0; i < D; ++i) {
            double s = 0.0;
            for (int n = 0; n < Ngeo; ++n) s += X[n * D + i] * ge(n, q);
            x[i] = s;
        }
    };

#pragma omp parallel for schedule(static)
    for (int64_t el = 0; el < E; ++el) {
        double J[9], Ji[9];
        double vol = 0.0;
        for (int q = 0; q < Nq; ++q) {
            jac(el, geoD_Q, Nq, q, J);
            double det = inv_det(D, J, Ji);
            double ad = std::fabs(det);
            vAbsDetJ[static_cast<std::size_t>(el) * Nq + q] = ad;
            // Ji[e * D + i] = (J^-1)_{e i} = d xi_e / d x_i
            for (int e = 0; e < D; ++e)
                for (int i = 0; i < D; ++i)
                    vG[(static_cast<std::size_t>(el) * DD + e * D + i) * Nq + q] = Ji[e * D + i];
            map(el, geoE_Q, q, &vCoords[(static_cast<std::size_t>(el) * Nq + q) * D]);
            vol += W[q] * ad;
        }
        volume[el] = vol;
    }

    // geometry at facet points (side 0 provides normal, coordinates and area)
    auto refN = reference_normals(D);
    fN.assign(static_cast<std::size_t>(F) * D * nq, 0.0);
    fNunit.assign(static_cast<std::size_t>(F) * D * nq, 0.0);
    fNl.assign(static_cast<std::size_t>(F) * nq, 0.0);
    fG0.assign(static_cast<std::size_t>(F) * DD * nq, 0.0);
    fG1.assign(static_cast<std::size_t>(F) * DD * nq, 0.0);
    fCoords.assign(static_cast<std::size_t>(F) * nq * D, 0.0);
    area.assign(F, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F; ++f) {
        double J[9], Ji[9];
        int64_t e0 = up[2 * f], e1 = up[2 * f + 1];
        int l0 = loc[2 * f], l1 = loc[2 * f + 1];
        double a = 0.0;
        for (int q = 0; q < nq; ++q) {
            jac(e0, geoD_q[l0], nq, q, J);
            double det = inv_det(D, J, Ji);
            // n_i = |det J| sum_j (J^-1)_{j i} N_j (Curvilinear::normal)
            double nl2 = 0.0;
            double n[3];
            for (int i = 0; i < D; ++i) {
                double s = 0.0;
                for (int j = 0; j < D; ++j) s += Ji[j * D + i] * refN[l0][j];
                n[i] = std::fabs(det) * s;
                nl2 += n[i] * n[i];
            }
            double nl = std::sqrt(nl2);
            for (int i = 0; i < D; ++i) {
                fN[(static_cast<std::size_t>(f) * D + i) * nq + q] = n[i];
                fNunit[(static_cast<std::size_t>(f) * D + i) * nq + q] = n[i] / nl;
            }
            fNl[static_cast<std::size_t>(f) * nq + q] = nl;
            a += w[q] * nl;
            for (int e = 0; e < D; ++e)
                for (int i = 0; i < D; ++i)
                    fG0[(static_cast<std::size_t>(f) * DD + e * D + i) * nq + q] = Ji[e * D + i];
            map(e0, geoE_q[l0], q, &fCoords[(static_cast<std::size_t>(f) * nq + q) * D]);
            jac(e1, geoD_q[l1], nq, q, J);
            inv_det(D, J, Ji);
            for (int e = 0; e < D; ++e)
                for (int i = 0; i < D; ++i)
                    fG1[(static_cast<std::size_t>(f) * DD + e * D + i) * nq + q] = Ji[e * D + i];
        }
        area[f] = a;
    }
    has_material = false;
    default_density();
}

void HostOperator::default_density() {
    Minv_ref = invert(space.mass_matrix());
    nrwj.assign(static_cast<std::size_t>(E) * Nq, 0.0);
    for (int64_t el = 0; el < E; ++el)
        for (int q = 0; q < Nq; ++q)
            nrwj[static_cast<std::size_t>(el) * Nq + q] = -W[q] / vAbsDetJ[static_cast<std::size_t>(el) * Nq + q];
}

// 1/rho at the volume points projected onto the nodal material space like lam and mu
// (project_material_rhs, app/kernels/elasticity.py:38-42), then evaluated at the points.
void HostOperator::set_density(double const* rho_Q) {
    if (!rho_Q) throw std::invalid_argument("density missing");
    if (Minv_ref.rows == 0) default_density();
    int nm = mat_space.num_basis();
#pragma omp parallel for schedule(static)
    for (int64_t el = 0; el < E; ++el) {
        Dense M(nm, nm);
        double const* J = &vAbsDetJ[static_cast<std::size_t>(el) * Nq];
        for (int k = 0; k < nm; ++k)
            for (int l = 0; l < nm; ++l) {
                double s = 0.0;
                for (int q = 0; q < Nq; ++q) s += matE_Q(k, q) * W[q] * J[q] * matE_Q(l, q);
                M(k, l) = s;
            }
        std::vector<double> b(nm);
        for (int k = 0; k < nm; ++k) {
            double s = 0.0;
            for (int q = 0; q < Nq; ++q) s += (1.0 / rho_Q[static_cast<std::size_t>(el) * Nq + q]) * matE_Q(k, q) * W[q] * J[q];
            b[k] = s;
        }
        solve_in_place(M, b.data());
        for (int q = 0; q < Nq; ++q) {
            double ri = 0.0;
            for (int t = 0; t < nm; ++t) ri += matE_Q(t, q) * b[t];
            nrwj[static_cast<std::size_t>(el) * Nq + q] = -ri * W[q] / J[q];
        }
    }
}

void HostOperator::set_material(double const* c0_Q, double const* c1_Q) {
    if (!c0_Q || (kind != kPoisson && !c1_Q)) throw std::invalid_argument("material missing");
    int nm = mat_space.num_basis();
    int DD = D * D;
    mat_nodal.assign(static_cast<std::size_t>(E) * 2 * nm, 0.0);
    vCoef.assign(static_cast<std::size_t>(E) * ncoef * Nq, 0.0);

    // L2 projection onto the nodal space (project_K_lhs/rhs, project_material_lhs/rhs)
#pragma omp parallel for schedule(static)
    for (int64_t el = 0; el < E; ++el) {
        Dense M(nm, nm);
        double const* J = &vAbsDetJ[static_cast<std::size_t>(el) * Nq];
        for (int k = 0; k < nm; ++k)
            for (int l = 0; l < nm; ++l) {
                double s = 0.0;
                for (int q = 0; q < Nq; ++q) s += matE_Q(k, q) * W[q] * J[q] * matE_Q(l, q);
                M(k, l) = s;
            }
        for (int c = 0; c < (kind == kPoisson ? 1 : 2); ++c) {
            double const* cq = (c == 0 ? c0_Q : c1_Q) + static_cast<std::size_t>(el) * Nq;
            std::vector<double> b(nm);
            for (int k = 0; k < nm; ++k) {
                double s = 0.0;
                for (int q = 0; q < Nq; ++q) s += cq[q] * matE_Q(k, q) * W[q] * J[q];
                b[k] = s;
            }
            solve_in_place(M, b.data());
            std::copy(b.begin(), b.end(), &mat_nodal[(static_cast<std::size_t>(el) * 2 + c) * nm]);
        }
        // volume coefficients at Q: Poisson |J| W K(x_q); Elasticity lam W |J|, mu W |J|
        for (int c = 0; c < ncoef; ++c) {
            double const* m = &mat_nodal[(static_cast<std::size_t>(el) * 2 + c) * nm];
            for (int q = 0; q < Nq; ++q) {
                double s = 0.0;
                for (int t = 0; t < nm; ++t) s += matE_Q(t, q) * m[t];
                vCoef[(static_cast<std::size_t>(el) * ncoef + c) * Nq + q] = s * W[q] * J[q];
            }
        }
    }

    // facet coefficients
    if (kind == kPoisson) {
        fCoef.assign(static_cast<std::size_t>(F) * 2 * DD * nq, 0.0);
    } else {
        fCoef.assign(static_cast<std::size_t>(F) * 4 * nq, 0.0);
    }
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F; ++f) {
        for (int s = 0; s < 2; ++s) {
            int64_t el = up[2 * f + s];
            Dense const& mE = matE_qf[loc[2 * f + s]];
            std::vector<double> const& G = (s == 0) ? fG0 : fG1;
            for (int q = 0; q < nq; ++q) {
                double v[2] = {0.0, 0.0};
                for (int c = 0; c < ncoef; ++c) {
                    double const* m = &mat_nodal[(static_cast<std::size_t>(el) * 2 + c) * nm];
                    double acc = 0.0;
                    for (int t = 0; t < nm; ++t) acc += mE(t, q) * m[t];
                    v[c] = acc;
                }
                if (kind == kPoisson) {
                    // K_G_q = K(x_q) G_q (kernel K_G_q, Poisson.cpp:167-193)
                    for (int c = 0; c < DD; ++c)
                        fCoef[((static_cast<std::size_t>(f) * 2 + s) * DD + c) * nq + q] =
                            v[0] * G[(static_cast<std::size_t>(f) * DD + c) * nq + q];
                } else {
                    fCoef[(static_cast<std::size_t>(f) * 4 + 2 * s + 0) * nq + q] = v[0];
                    fCoef[(static_cast<std::size_t>(f) * 4 + 2 * s + 1) * nq + q] = v[1];
                }
            }
        }
    }

    // interior penalty (prepare_penalty): p(side) = (D+1) c_{N-1} |f|/|E| c1^2/c0,
    // interior (p0 + p1)/4, boundary p0.
    penalty.assign(F, 0.0);
    double cN1 = trace_constant(D, N - 1);
    auto bounds = [&](int64_t el, double& c0, double& c1) {
        double const* a = &mat_nodal[(static_cast<std::size_t>(el) * 2 + 0) * nm];
        double const* b = &mat_nodal[(static_cast<std::size_t>(el) * 2 + 1) * nm];
        c0 = std::numeric_limits<double>::max();
        c1 = std::numeric_limits<double>::lowest();
        for (int i = 0; i < nm; ++i) {
            if (kind == kPoisson) {
                c0 = std::min(c0, a[i]);
                c1 = std::max(c1, a[i]);
            } else {
                c0 = std::min(c0, 2.0 * b[i]);
                c1 = std::max(c1, D * a[i] + 2.0 * b[i]);
            }
        }
    };
    for (int64_t f = 0; f < F; ++f) {
        auto p = [&](int s) {
            int64_t el = up[2 * f + s];
            double c0, c1;
            bounds(el, c0, c1);
            return (D + 1) * cN1 * (area[f] / volume[el]) * (c1 * c1 / c0);
        };
        penalty[f] = (up[2 * f] != up[2 * f + 1]) ? (p(0) + p(1)) / 4.0 : p(0);
    }
    has_material = true;
}

void HostOperator::rhs(double const* force_Q, double const* bc_q, double* b) const {
    if (!has_material) throw std::logic_error("rhs before set_material");
    int DD = D * D;
    std::fill(b, b + static_cast<std::size_t>(E) * bs, 0.0);
    if (force_Q) {
#pragma omp parallel for schedule(static)
        for (int64_t el = 0; el < E; ++el) {
            double const* J = &vAbsDetJ[static_cast<std::size_t>(el) * Nq];
            for (int p = 0; p < Q; ++p) {
                double const* Fq = force_Q + (static_cast<std::size_t>(el) * Q + p) * Nq;
                for (int k = 0; k < Nbf; ++k) {
                    double s = 0.0;
                    for (int q = 0; q < Nq; ++q) s += J[q] * W[q] * E_Q(k, q) * Fq[q];
                    b[static_cast<std::size_t>(el) * bs + k + Nbf * p] += s;
                }
            }
        }
    }
    if (!bc_q) return;
    constexpr double eps = -1.0;  // SIPG
    // facet terms: serial over facets (elements may be touched by several facets)
    std::vector<double> fq(static_cast<std::size_t>(Q) * nq), flift(static_cast<std::size_t>(Q) * nq);
    std::vector<double> Dx(static_cast<std::size_t>(Nbf) * D * nq);
    for (int64_t f = 0; f < F; ++f) {
        int fbc = bc[f];
        if (fbc != 3 && fbc != 5) continue;
        bool boundary = up[2 * f] == up[2 * f + 1];
        for (int i = 0; i < Q * nq; ++i) {
            fq[i] = bc_q[static_cast<std::size_t>(f) * Q * nq + i];
            // bc_boundary halves slip on a boundary fault facet (Poisson.cpp:418-432)
            if (boundary && fbc == 3) fq[i] *= 0.5;
        }
        // IP lift: f_lifted_q = nl_q f_q
        for (int p = 0; p < Q; ++p)
            for (int q = 0; q < nq; ++q)
                flift[p * nq + q] = fNl[static_cast<std::size_t>(f) * nq + q] * fq[p * nq + q];
        int nsides = boundary ? 1 : 2;
        for (int s = 0; s < nsides; ++s) {
            double c10 = boundary ? eps : 0.5 * eps;
            double c20 = (s == 0) ? penalty[f] : -penalty[f];
            int64_t el = up[2 * f + s];
            int l = loc[2 * f + s];
            Dense const& Eq = E_qf[l];
            std::vector<double> const& Dxi = Dxi_qf[l];
            std::vector<double> const& G = (s == 0) ? fG0 : fG1;
            // Dx[k][i][q] = sum_e G(e,i) Dxi[k][e][q]
            for (int k = 0; k < Nbf; ++k)
                for (int i = 0; i < D; ++i)
                    for (int q = 0; q < nq; ++q) {
                        double acc = 0.0;
                        for (int e = 0; e < D; ++e)
                            acc += G[(static_cast<std::size_t>(f) * DD + e * D + i) * nq + q] *
                                   Dxi[(static_cast<std::size_t>(k) * D + e) * nq + q];
                        Dx[(static_cast<std::size_t>(k) * D + i) * nq + q] = acc;
                    }
            double const* n = &fN[static_cast<std::size_t>(f) * D * nq];
            double* bb = b + static_cast<std::size_t>(el) * bs;
            if (kind == kPoisson) {
                // K_q of this side from K*G: recompute K(x_q) = matE . K
                int nm = mat_space.num_basis();
                double const* K = &mat_nodal[(static_cast<std::size_t>(el) * 2) * nm];
                for (int k = 0; k < Nbf; ++k) {
                    double s1 = 0.0, s2 = 0.0;
                    for (int q = 0; q < nq; ++q) {
                        double Kq = 0.0;
                        for (int t = 0; t < nm; ++t) Kq += matE_qf[l](t, q) * K[t];
                        double dn = 0.0;
                        for (int i = 0; i < D; ++i)
                            dn += Kq * Dx[(static_cast<std::size_t>(k) * D + i) * nq + q] * n[i * nq + q];
                        s1 += w[q] * dn * fq[q];
                        s2 += w[q] * Eq(k, q) * flift[q];
                    }
                    bb[k] += c10 * s1 + c20 * s2;
                }
            } else {
                double const* lam = &fCoef[(static_cast<std::size_t>(f) * 4 + 2 * s + 0) * nq];
                double const* mu = &fCoef[(static_cast<std::size_t>(f) * 4 + 2 * s + 1) * nq];
                for (int k = 0; k < Nbf; ++k)
                    for (int p = 0; p < Q; ++p) {
                        double s1 = 0.0, s2 = 0.0;
                        for (int q = 0; q < nq; ++q) {
                            double un = 0.0, dxn = 0.0, dxu = 0.0;
                            for (int i = 0; i < D; ++i) {
                                un += fq[i * nq + q] * n[i * nq + q];
                                dxn += Dx[(static_cast<std::size_t>(k) * D + i) * nq + q] * n[i * nq + q];
                                dxu += Dx[(static_cast<std::size_t>(k) * D + i) * nq + q] * fq[i * nq + q];
                            }
                            double dkp = Dx[(static_cast<std::size_t>(k) * D + p) * nq + q];
                            double tt = lam[q] * dkp * un + mu[q] * (dxn * fq[p * nq + q] + dxu * n[p * nq + q]);
                            s1 += w[q] * tt;
                            s2 += w[q] * Eq(k, q) * flift[p * nq + q];
                        }
                        bb[k + Nbf * p] += c10 * s1 + c20 * s2;
                    }
            }
        }
    }
}

int64_t HostOperator::flops_apply() const {
    // Algorithmic FLOPs with each facet flux evaluated once (FMA = 2 FLOP).
    int64_t vol, fct;
    if (kind == kPoisson) {
        vol = 4LL * Nbf * D * Nq + 4LL * D * D * Nq + D * Nq;
        fct = 8LL * Nbf * nq + 8LL * Nbf * D * nq + 8LL * D * D * nq + (11LL * D + 4) * nq;
    } else {
        vol = 4LL * Nbf * D * Nq * Q + 4LL * D * D * Nq * Q + (3LL * D * D + D + 2) * Nq;
        fct = 8LL * Nbf * Q * nq + 8LL * Nbf * D * Q * nq + 8LL * D * D * Q * nq +
              (18LL * D * D + 9LL * D + 2LL * Q + 4LL * D * Q) * nq;
    }
    int64_t total = vol * E;
    for (int64_t f = 0; f < F; ++f) {
        bool boundary = up[2 * f] == up[2 * f + 1];
        if (!boundary) {
            if (bc[f] != 1) total += fct;
        } else if (bc[f] == 3 || bc[f] == 5) {
            total += fct / 2;
        }
    }
    return total;
}

int64_t HostOperator::bytes_apply(int s) const {
    int64_t per_el = 2LL * bs + static_cast<int64_t>(D) * D * Nq + static_cast<int64_t>(ncoef) * Nq;
    int64_t per_f = (kind == kPoisson)
                        ? (static_cast<int64_t>(D) * nq + nq + 2LL * D * D * nq + 1)
                        : (static_cast<int64_t>(D) * nq + nq + 4LL * nq + 2LL * D * D * nq + 1);
    return E * per_el * s + F * (per_f * s + 20);
}

// ---- error norms at a caller-chosen rule --------------------------------------------------------

namespace {

// Geometry of element el at the rule's points: |det J| and J^-1 (Ji[e * D + i] = d xi_e / d x_i).
void rule_geometry(HostOperator const& h, int64_t el, std::vector<double> const& gd, int np, int q, double* Ji,
                   double* absdet) {
    const int D = h.D;
    double const* X = &h.geo_nodes[static_cast<std::size_t>(el) * h.Ngeo * D];
    double J[9];
    for (int i = 0; i < D; ++i)
        for (int e = 0; e < D; ++e) {
            double acc = 0.0;
            for (int n = 0; n < h.Ngeo; ++n) acc += X[n * D + i] * gd[(static_cast<std::size_t>(n) * D + e) * np + q];
            J[i * D + e] = acc;
        }
    *absdet = std::fabs(inv_det(D, J, Ji));
}

}  // namespace

void HostOperator::rule_coords(int np, double const* pts, double* out) const {
    Dense ge = geo_space.eval(Points(pts, pts + static_cast<std::size_t>(np) * D));
#pragma omp parallel for schedule(static)
    for (int64_t el = 0; el < E; ++el) {
        double const* X = &geo_nodes[static_cast<std::size_t>(el) * Ngeo * D];
        for (int q = 0; q < np; ++q)
            for (int i = 0; i < D; ++i) {
                double acc = 0.0;
                for (int n = 0; n < Ngeo; ++n) acc += X[n * D + i] * ge(n, q);
                out[(static_cast<std::size_t>(el) * np + q) * D + i] = acc;
            }
    }
}

void HostOperator::project(double const* U_Q, double* y) const {
    const int nb = Nbf;
#pragma omp parallel for schedule(static)
    for (int64_t el = 0; el < E; ++el) {
        double const* J = &vAbsDetJ[static_cast<std::size_t>(el) * Nq];
        std::vector<double> u(static_cast<std::size_t>(nb)), t(static_cast<std::size_t>(nb)),
            v(static_cast<std::size_t>(Nq)), r(static_cast<std::size_t>(nb));
        for (int p = 0; p < Q; ++p) {
            double const* f = &U_Q[(static_cast<std::size_t>(el) * Q + p) * Nq];
            for (int k = 0; k < nb; ++k) {  // U = E_Q W |J| U_Q
                double acc = 0.0;
                for (int q = 0; q < Nq; ++q) acc += E_Q(k, q) * W[q] * J[q] * f[q];
                u[k] = acc;
            }
            for (int s = 0; s < nb; ++s) {  // MinvRef U
                double acc = 0.0;
                for (int l = 0; l < nb; ++l) acc += Minv_ref(s, l) * u[l];
                t[s] = acc;
            }
            for (int q = 0; q < Nq; ++q) {  // (W / |J|) E_Q^T (MinvRef U)
                double acc = 0.0;
                for (int s = 0; s < nb; ++s) acc += E_Q(s, q) * t[s];
                v[q] = W[q] / J[q] * acc;
            }
            for (int rr = 0; rr < nb; ++rr) {
                double acc = 0.0;
                for (int q = 0; q < Nq; ++q) acc += E_Q(rr, q) * v[q];
                r[rr] = acc;
            }
            for (int k = 0; k < nb; ++k) {  // MinvRef (...)
                double acc = 0.0;
                for (int rr = 0; rr < nb; ++rr) acc += Minv_ref(k, rr) * r[rr];
                y[el * bs + k + p * nb] = acc;
            }
        }
    }
}

void HostOperator::evaluate(double const* x, int np, double const* pts, double* out) const {
    Dense Eb = space.eval(Points(pts, pts + static_cast<std::size_t>(np) * D));
#pragma omp parallel for schedule(static)
    for (int64_t el = 0; el < E; ++el)
        for (int p = 0; p < Q; ++p)
            for (int q = 0; q < np; ++q) {
                double acc = 0.0;
                for (int k = 0; k < Nbf; ++k) acc += Eb(k, q) * x[el * bs + k + p * Nbf];
                out[(static_cast<std::size_t>(el) * Q + p) * np + q] = acc;
            }
}

double HostOperator::error_l2(double const* x, int np, double const* pts, double const* w, double const* ref) const {
    Points P(pts, pts + static_cast<std::size_t>(np) * D);
    Dense Eb = space.eval(P);
    std::vector<double> gd = geo_space.grad(P);
    std::vector<double> part(static_cast<std::size_t>(E), 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t el = 0; el < E; ++el) {
        double acc = 0.0;
        for (int q = 0; q < np; ++q) {
            double Ji[9], ad;
            rule_geometry(*this, el, gd, np, q, Ji, &ad);
            for (int j = 0; j < Q; ++j) {
                double u = 0.0;
                for (int k = 0; k < Nbf; ++k) u += Eb(k, q) * x[el * bs + k + j * Nbf];
                const double e = ref[(static_cast<std::size_t>(el) * Q + j) * np + q] - u;
                acc += w[q] * ad * e * e;
            }
        }
        part[static_cast<std::size_t>(el)] = acc;
    }
    double err = 0.0;
    for (double v : part) err += v;
    return std::sqrt(err);
}

double HostOperator::error_h1_semi(double const* x, int np, double const* pts, double const* w,
                                   double const* refgrad) const {
    Points P(pts, pts + static_cast<std::size_t>(np) * D);
    std::vector<double> Gb = space.grad(P);  // [(k * D + e) * np + q]
    std::vector<double> gd = geo_space.grad(P);
    std::vector<double> part(static_cast<std::size_t>(E), 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t el = 0; el < E; ++el) {
        double acc = 0.0;
        for (int q = 0; q < np; ++q) {
            double Ji[9], ad;
            rule_geometry(*this, el, gd, np, q, Ji, &ad);
            for (int j = 0; j < Q; ++j)
                for (int d = 0; d < D; ++d) {
                    double g = 0.0;
                    for (int k = 0; k < Nbf; ++k) {
                        double dx = 0.0;
                        for (int e = 0; e < D; ++e) dx += Ji[e * D + d] * Gb[(static_cast<std::size_t>(k) * D + e) * np + q];
                        g += dx * x[el * bs + k + j * Nbf];
                    }
                    const double e = refgrad[((static_cast<std::size_t>(el) * Q + j) * D + d) * np + q] - g;
                    acc += w[q] * ad * e * e;
                }
        }
        part[static_cast<std::size_t>(el)] = acc;
    }
    double err = 0.0;
    for (double v : part) err += v;
    return std::sqrt(err);
}

// ---- p-multigrid set-up ----------------------------------------------------------------------

Dense interpolation_matrix(int D, int kind, int n_to, int n_from) {
    if (n_to <= n_from || n_from < 0) throw std::invalid_argument("interpolation needs n_to > n_from >= 0");
    const int N1 = num_basis(D, n_to), N2 = num_basis(D, n_from);
    Dense I(N1, N2);
    if (kind == kPoisson) {
        // graded Dubiner ordering: the first N2 modal functions span the degree-n_from space
        for (int l = 0; l < N2; ++l) I(l, l) = 1.0;
        return I;
    }
    RefSpace coarse = RefSpace::nodal(D, n_from, warp_blend_nodes(D, n_from));
    Dense Ec = coarse.eval(warp_blend_nodes(D, n_to));  // [N2][N1]: coarse basis l at fine node k
    for (int k = 0; k < N1; ++k)
        for (int l = 0; l < N2; ++l) I(k, l) = Ec(l, k);
    return I;
}

std::vector<int> mg_level_degrees(int strategy, int coarse, int N) {
    if (N <= coarse) coarse = N > 0 ? N - 1 : 0;
    std::vector<int> lv;
    if (strategy == 0) {
        lv = {coarse, N};
    } else if (strategy == 1) {
        lv.push_back(N);
        while (lv.back() > coarse) lv.push_back(lv.back() / 2);
        if (lv.back() != coarse) lv.back() = coarse;
        std::reverse(lv.begin(), lv.end());
    } else if (strategy == 2) {
        for (int d = coarse; d <= N; ++d) lv.push_back(d);
    } else {
        throw std::invalid_argument("unknown multigrid strategy");
    }
    return lv;
}

std::vector<int32_t> element_neighbours(HostOperator const& h) {
    const int NB = 1 + h.nfaces;
    std::vector<int32_t> nbr(static_cast<size_t>(h.E) * NB, -1);
    for (int64_t e = 0; e < h.E; ++e) {
        nbr[static_cast<size_t>(e) * NB] = static_cast<int32_t>(e);
        for (int f = 0; f < h.nfaces; ++f) {
            const Side& s = h.sides[static_cast<size_t>(e) * h.nfaces + f];
            if (s.nb != e) nbr[static_cast<size_t>(e) * NB + 1 + f] = s.nb;
        }
    }
    return nbr;
}

std::vector<int32_t> distance2_colouring(std::vector<int32_t> const& nbr, int64_t E, int NB, int* ncolors) {
    std::vector<int32_t> col(static_cast<size_t>(E), -1);
    std::vector<int64_t> stamp;  // stamp[c] == e: colour c is taken near element e
    int nc = 0;
    for (int64_t e = 0; e < E; ++e) {
        auto mark = [&](int32_t t) {
            if (t >= 0 && col[t] >= 0) stamp[col[t]] = e;
        };
        for (int a = 0; a < NB; ++a) {
            const int32_t n = nbr[static_cast<size_t>(e) * NB + a];
            if (n < 0) continue;
            mark(n);
            for (int b = 1; b < NB; ++b) mark(nbr[static_cast<size_t>(n) * NB + b]);
        }
        int c = 0;
        while (c < nc && stamp[c] == e) ++c;
        if (c == nc) {
            stamp.push_back(-1);
            ++nc;
        }
        col[e] = c;
    }
    *ncolors = nc;
    return col;
}

std::vector<int32_t> vertex_numbering(HostOperator const& h, int64_t* nv) {
    const int NV = h.D + 1;
    const int64_t n = h.E * NV;
    std::vector<int64_t> parent(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) parent[static_cast<size_t>(i)] = i;
    auto find = [&](int64_t a) {
        while (parent[static_cast<size_t>(a)] != a) {
            parent[static_cast<size_t>(a)] = parent[static_cast<size_t>(parent[static_cast<size_t>(a)])];
            a = parent[static_cast<size_t>(a)];
        }
        return a;
    };
    auto fv = facet_vertices(h.D);
    for (int64_t f = 0; f < h.F; ++f) {
        const int64_t e0 = h.up[static_cast<size_t>(2 * f)], e1 = h.up[static_cast<size_t>(2 * f + 1)];
        if (e0 == e1) continue;
        const int l0 = h.loc[static_cast<size_t>(2 * f)], l1 = h.loc[static_cast<size_t>(2 * f + 1)];
        for (int k = 0; k < h.D; ++k) {
            int64_t a = find(e0 * NV + fv[static_cast<size_t>(l0)][static_cast<size_t>(k)]);
            int64_t b = find(e1 * NV + fv[static_cast<size_t>(l1)][static_cast<size_t>(k)]);
            if (a != b) parent[static_cast<size_t>(std::max(a, b))] = std::min(a, b);
        }
    }
    std::vector<int32_t> vid(static_cast<size_t>(n));
    std::vector<int32_t> id_of_root(static_cast<size_t>(n), -1);
    int32_t next = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int64_t r = find(i);
        if (id_of_root[static_cast<size_t>(r)] < 0) id_of_root[static_cast<size_t>(r)] = next++;
        vid[static_cast<size_t>(i)] = id_of_root[static_cast<size_t>(r)];
    }
    *nv = next;
    return vid;
}

Dense linear_to_space(int D, int kind, int p) {
    Points nodes = warp_blend_nodes(D, p);
    RefSpace sp = (kind == kPoisson) ? RefSpace::modal(D, p) : RefSpace::nodal(D, p, nodes);
    Dense Eb = sp.eval(nodes);  // [Nbf][Nnodes]
    const int nb = Eb.rows;
    Dense V(nb, nb);
    for (int j = 0; j < nb; ++j)
        for (int k = 0; k < nb; ++k) V(j, k) = Eb(k, j);
    Dense Vi = invert(V);
    Dense T(nb, D + 1);
    for (int j = 0; j < nb; ++j) {
        const double* x = &nodes[static_cast<size_t>(j) * D];
        double lam[4];
        lam[0] = 1.0;
        for (int d = 0; d < D; ++d) {
            lam[d + 1] = x[d];
            lam[0] -= x[d];
        }
        for (int k = 0; k < nb; ++k)
            for (int i = 0; i <= D; ++i) T(k, i) += Vi(k, j) * lam[i];
    }
    return T;
}

VertexCsr vertex_galerkin(std::vector<double> const& A, std::vector<int32_t> const& nbr, int64_t E, int NB, int D,
                          int Nbf, int Q, Dense const& T, std::vector<int32_t> const& vid, int64_t nv) {
    const int NV = D + 1, bs = Nbf * Q, m = NV * Q;
    VertexCsr c;
    c.nv = nv;
    c.Q = Q;
    // sparsity: every (corner of e, corner of t) pair of a present block (e, s)
    std::vector<int64_t> keys;
    keys.reserve(static_cast<size_t>(E) * NB * NV * NV);
    for (int64_t e = 0; e < E; ++e)
        for (int s = 0; s < NB; ++s) {
            const int32_t t = nbr[static_cast<size_t>(e * NB + s)];
            if (t < 0) continue;
            for (int i = 0; i < NV; ++i)
                for (int j = 0; j < NV; ++j)
                    keys.push_back(static_cast<int64_t>(vid[static_cast<size_t>(e * NV + i)]) * nv +
                                   vid[static_cast<size_t>(static_cast<int64_t>(t) * NV + j)]);
        }
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    c.ptr.assign(static_cast<size_t>(nv) + 1, 0);
    c.col.resize(keys.size());
    for (size_t k = 0; k < keys.size(); ++k) {
        ++c.ptr[static_cast<size_t>(keys[k] / nv) + 1];
        c.col[k] = static_cast<int32_t>(keys[k] % nv);
    }
    for (int64_t v = 0; v < nv; ++v) c.ptr[static_cast<size_t>(v) + 1] += c.ptr[static_cast<size_t>(v)];
    c.val.assign(keys.size() * Q * Q, 0.0);
    // values: B = R_e^T A_es R_t per block, scattered by vertex pair
    std::vector<double> AT(static_cast<size_t>(bs) * m), B(static_cast<size_t>(m) * m);
    for (int64_t e = 0; e < E; ++e)
        for (int s = 0; s < NB; ++s) {
            const int32_t t = nbr[static_cast<size_t>(e * NB + s)];
            if (t < 0) continue;
            const double* a = &A[static_cast<size_t>((e * NB + s) * bs) * bs];  // a[col * bs + row]
            // AT[row][(j, q)] = sum_k' A[row][k' + q Nbf] T(k', j)
            for (int row = 0; row < bs; ++row)
                for (int q = 0; q < Q; ++q)
                    for (int j = 0; j < NV; ++j) {
                        double acc = 0.0;
                        for (int kk = 0; kk < Nbf; ++kk) acc += a[static_cast<size_t>(kk + q * Nbf) * bs + row] * T(kk, j);
                        AT[static_cast<size_t>(row) * m + j * Q + q] = acc;
                    }
            // B[(i, p)][(j, q)] = sum_k T(k, i) AT[k + p Nbf][(j, q)]
            for (int i = 0; i < NV; ++i)
                for (int p = 0; p < Q; ++p)
                    for (int jq = 0; jq < m; ++jq) {
                        double acc = 0.0;
                        for (int k = 0; k < Nbf; ++k) acc += T(k, i) * AT[static_cast<size_t>(k + p * Nbf) * m + jq];
                        B[static_cast<size_t>(i * Q + p) * m + jq] = acc;
                    }
            for (int i = 0; i < NV; ++i) {
                const int64_t v = vid[static_cast<size_t>(e * NV + i)];
                const int32_t* c0 = c.col.data() + c.ptr[static_cast<size_t>(v)];
                const int32_t* c1 = c.col.data() + c.ptr[static_cast<size_t>(v) + 1];
                for (int j = 0; j < NV; ++j) {
                    const int32_t w = vid[static_cast<size_t>(static_cast<int64_t>(t) * NV + j)];
                    const size_t pos = static_cast<size_t>(std::lower_bound(c0, c1, w) - c.col.data());
                    double* out = &c.val[pos * Q * Q];
                    for (int p = 0; p < Q; ++p)
                        for (int q = 0; q < Q; ++q) out[p * Q + q] += B[static_cast<size_t>(i * Q + p) * m + j * Q + q];
                }
            }
        }
    // incidences (element, corner) per vertex
    c.vinc_ptr.assign(static_cast<size_t>(nv) + 1, 0);
    for (int64_t k = 0; k < E * NV; ++k) ++c.vinc_ptr[static_cast<size_t>(vid[static_cast<size_t>(k)]) + 1];
    for (int64_t v = 0; v < nv; ++v) c.vinc_ptr[static_cast<size_t>(v) + 1] += c.vinc_ptr[static_cast<size_t>(v)];
    c.vinc.resize(static_cast<size_t>(E * NV));
    std::vector<int64_t> fill(c.vinc_ptr.begin(), c.vinc_ptr.end() - 1);
    for (int64_t k = 0; k < E * NV; ++k)
        c.vinc[static_cast<size_t>(fill[static_cast<size_t>(vid[static_cast<size_t>(k)])]++)] = static_cast<int32_t>(k);
    return c;
}

}  // namespace tdg
