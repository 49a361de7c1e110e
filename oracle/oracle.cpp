// ORACLE -- test infrastructure only.  A CPU restatement of tandem's matrix-free DG operator in
// tandem's own element-centric form and data layout, used by tests/, the smoke check and the CPU
// baseline of bench.py as the checker.  Nothing in the product links or calls it.
//
// Followed, routine by routine:
//   geometry   DGCurvilinearCommon::prepare_volume / prepare_bndskl
//              (src/form/DGCurvilinearCommon.cpp:41-102), Curvilinear::jacobian / jacobianInv /
//              detJ / normal / map (src/geometry/Curvilinear.cpp:174-274)
//   topology   DGOperatorTopo (src/form/DGOperatorTopo.cpp:46-85): SideInfo per element face
//   Poisson    prepare_volume / prepare_skeleton / prepare_boundary / prepare_volume_post_skeleton /
//              prepare_penalty (app/localoperator/Poisson.cpp:133-223); apply (Poisson.cpp:551-644)
//              with the einsums of app/kernels/poisson.py:120-140; assemble_volume / skeleton /
//              boundary (Poisson.cpp:225-385, poisson.py:30-75); rhs_* (Poisson.cpp:387-549)
//   Elasticity prepare_* (app/localoperator/Elasticity.cpp:104-292); apply_<false>
//              (Elasticity.cpp:698-863) with app/kernels/elasticity.py:181-234; assemble_*
//              (Elasticity.cpp:317-519, elasticity.py:55-149); rhs_* (Elasticity.cpp:521-696)
//   loops      DGOperator::apply_ / assemble / rhs (src/form/DGOperator.h:121-237,363-396)
//   solver     preconditioned CG (PETSc KSPCG as configured by app/common/PetscLinearSolver.cpp:22-28)
//              with the element block-Jacobi preconditioner (PCPBJACOBI over the assembled P)
//   errors     Error<D>::L2 / H1_semi (src/form/Error.cpp) with the operator's volume rule
//   wave       the inverse mass of Elasticity::wave_rhs (app/localoperator/Elasticity.cpp:865-880,
//              app/kernels/elasticity.py:236-237) with negative_rhoInv_W_Jinv_Q of
//              precomputeVolume (elasticity.py:44-48) and 1/rho projected like lam and mu
//              (project_material_rhs, elasticity.py:38-42)
// The reference-element tables (Dubiner / warp & blend bases, nodes) come from the product's
// tdg::RefSpace, which the tests pin against tandem's own known-answer tests.
#include "../include/tandem_b200.h"
#include "../tandem_b200/csrc/host/refelem.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

using tdg::Dense;
using tdg::Points;
using tdg::RefSpace;

namespace {

enum { kPoisson = 0, kElasticity = 1 };
enum { BC_None = 0, BC_Natural = 1, BC_Fault = 3, BC_Dirichlet = 5 };

struct SideInfo {
    long fctNo;
    int side;
    long lid;
    int localNo;
    int bc;
};
struct FacetInfo {
    long up[2];
    int localNo[2];
    int bc;
};

}  // namespace

struct orc_op {
    int D, N, kind, Q, Nbf, bs, Nq, nq, NF, Ngeo;
    long E, F;
    std::vector<double> W, w;
    RefSpace space, mat, geo;
    // tandem tensors (column-major index order as in the YATeTo specs)
    std::vector<double> E_Q;                   // E_Q(k, q) at k + Nbf q
    std::vector<double> Dxi_Q;                 // Dxi_Q(k, e, q) at k + Nbf (e + D q)
    std::vector<std::vector<double>> E_q;      // E_q[f](k, q)
    std::vector<std::vector<double>> Dxi_q;    // Dxi_q[f](k, e, q)
    std::vector<double> matE_Q;                // matE_Q_T(q, m) at q + Nq m
    std::vector<std::vector<double>> matE_q;   // matE_q_T[f](q, m)
    std::vector<FacetInfo> fct;
    std::vector<SideInfo> sides;  // [E][NF]
    // per element volume data: JInv(e, i, q) at e + D (i + D q), AbsDetJ(q), Coords(d, q)
    std::vector<double> JInv, AbsDetJ, Coords, volume;
    // per facet: Normal(d, q), UnitNormal, NormalLength(q), JInv0/JInv1, Coords, area
    std::vector<double> Normal, UnitNormal, NormalLength, JInv0, JInv1, FCoords, area;
    // material (nodal), volume precompute, facet precompute, penalty
    std::vector<double> matA, matB;            // [E][Nbf] (Poisson K; Elasticity lam, mu)
    std::vector<double> vol0, vol1;            // Poisson J_W_K_Q; Elasticity lam_W_J_Q, mu_W_J_Q
    std::vector<double> KG0, KG1;              // Poisson K_G_q side 0/1 (e, i, q)
    std::vector<double> lam0, mu0, lam1, mu1;  // Elasticity facet material (q)
    std::vector<double> penalty;
    std::vector<double> rhoInv;                // Elasticity: nodal 1/rho [E][Nbf] (empty: rho = 1)
    bool ready = false;
    // block-Jacobi inverses
    std::vector<double> pc;
};

namespace {

inline long idx3(int a, int b, int c, int A, int B) { return a + static_cast<long>(A) * (b + static_cast<long>(B) * c); }

void inv_det(int D, const double* J, double* Ji, double* det) {
    // J(i, e) column-major: J[i + D e]
    Dense m(D, D);
    for (int i = 0; i < D; ++i)
        for (int e = 0; e < D; ++e) m(i, e) = J[i + D * e];
    Dense inv = tdg::invert(m);
    for (int i = 0; i < D; ++i)
        for (int e = 0; e < D; ++e) Ji[i + D * e] = inv(i, e);
    if (D == 2) {
        *det = m(0, 0) * m(1, 1) - m(0, 1) * m(1, 0);
    } else {
        *det = m(0, 0) * (m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1)) - m(0, 1) * (m(1, 0) * m(2, 2) - m(1, 2) * m(2, 0)) +
               m(0, 2) * (m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0));
    }
}

std::vector<double> to_colmajor(Dense const& m) {
    std::vector<double> out(static_cast<size_t>(m.rows) * m.cols);
    for (int i = 0; i < m.rows; ++i)
        for (int j = 0; j < m.cols; ++j) out[i + static_cast<size_t>(m.rows) * j] = m(i, j);
    return out;
}

// RefSpace::grad gives g[(k * D + e) * np + q]; tandem's Dxi(k, e, q) is k + Nbf (e + D q).
std::vector<double> grad_tandem(RefSpace const& s, Points const& pts, int D) {
    int np = static_cast<int>(pts.size() / D);
    int nbf = s.num_basis();
    auto g = s.grad(pts);
    std::vector<double> out(static_cast<size_t>(nbf) * D * np);
    for (int k = 0; k < nbf; ++k)
        for (int e = 0; e < D; ++e)
            for (int q = 0; q < np; ++q) out[idx3(k, e, q, nbf, D)] = g[(static_cast<size_t>(k) * D + e) * np + q];
    return out;
}

// Curvilinear::jacobian at np points for element el: J(i, e, q) = sum_n X(i, n) gradE(n, e, q)
void jacobian(orc_op const& op, std::vector<double> const& geo_nodes, long el, std::vector<double> const& gD, int np,
              double* J) {
    const int D = op.D;
    const double* X = &geo_nodes[static_cast<size_t>(el) * op.Ngeo * D];
    for (int q = 0; q < np; ++q)
        for (int e = 0; e < D; ++e)
            for (int i = 0; i < D; ++i) {
                double s = 0.0;
                for (int n = 0; n < op.Ngeo; ++n) s += X[n * D + i] * gD[idx3(n, e, q, op.Ngeo, D)];
                J[i + D * (e + D * q)] = s;
            }
}

}  // namespace

extern "C" {

int orc_create(const tdg_mesh_desc* m, const tdg_quadrature* qd, int kind, orc_op** out) {
    try {
        auto* op = new orc_op();
        const int D = m->dim;
        op->D = D;
        op->N = m->degree;
        op->kind = kind;
        op->Q = kind == kPoisson ? 1 : D;
        op->NF = D + 1;
        op->E = m->num_elements;
        op->F = m->num_facets;
        op->Nq = qd->num_vol_points;
        op->nq = qd->num_fct_points;
        op->W.assign(qd->vol_weights, qd->vol_weights + op->Nq);
        op->w.assign(qd->fct_weights, qd->fct_weights + op->nq);
        Points vx(qd->vol_points, qd->vol_points + static_cast<size_t>(op->Nq) * D);
        Points fx(qd->fct_points, qd->fct_points + static_cast<size_t>(op->nq) * (D - 1));
        auto wb = tdg::warp_blend_nodes(D, op->N);
        op->space = kind == kPoisson ? RefSpace::modal(D, op->N) : RefSpace::nodal(D, op->N, wb);
        op->mat = RefSpace::nodal(D, op->N, wb);
        op->geo = RefSpace::nodal(D, m->geo_degree, tdg::warp_blend_nodes(D, m->geo_degree));
        op->Nbf = op->space.num_basis();
        op->bs = op->Nbf * op->Q;
        op->Ngeo = op->geo.num_basis();
        op->E_Q = to_colmajor(op->space.eval(vx));
        op->Dxi_Q = grad_tandem(op->space, vx, D);
        {
            Dense me = op->mat.eval(vx);  // (m, q) -> matE_Q_T(q, m)
            op->matE_Q.assign(static_cast<size_t>(op->Nq) * op->Nbf, 0.0);
            for (int mm = 0; mm < op->Nbf; ++mm)
                for (int q = 0; q < op->Nq; ++q) op->matE_Q[q + static_cast<size_t>(op->Nq) * mm] = me(mm, q);
        }
        std::vector<Points> fp(op->NF);
        for (int f = 0; f < op->NF; ++f) {
            fp[f] = tdg::facet_param(D, f, fx);
            op->E_q.push_back(to_colmajor(op->space.eval(fp[f])));
            op->Dxi_q.push_back(grad_tandem(op->space, fp[f], D));
            Dense me = op->mat.eval(fp[f]);
            std::vector<double> t(static_cast<size_t>(op->nq) * op->Nbf);
            for (int mm = 0; mm < op->Nbf; ++mm)
                for (int q = 0; q < op->nq; ++q) t[q + static_cast<size_t>(op->nq) * mm] = me(mm, q);
            op->matE_q.push_back(t);
        }
        // topology
        op->fct.resize(op->F);
        op->sides.assign(static_cast<size_t>(op->E) * op->NF, SideInfo{-1, 0, -1, 0, 0});
        for (long f = 0; f < op->F; ++f) {
            FacetInfo& fi = op->fct[f];
            for (int s = 0; s < 2; ++s) {
                fi.up[s] = m->facet_up[2 * f + s];
                fi.localNo[s] = m->facet_local_no[2 * f + s];
            }
            fi.bc = m->facet_bc[f];
            for (int i = 0; i < 2; ++i) {
                SideInfo& si = op->sides[fi.up[i] * op->NF + fi.localNo[i]];
                si.fctNo = f;
                si.side = i;
                si.lid = fi.up[(i + 1) % 2];
                si.localNo = fi.localNo[(i + 1) % 2];
                si.bc = fi.bc;
            }
        }
        // geometry
        std::vector<double> geo_nodes(m->geo_nodes, m->geo_nodes + static_cast<size_t>(op->E) * op->Ngeo * D);
        auto geoD_Q = grad_tandem(op->geo, vx, D);
        Dense geoE_Q = op->geo.eval(vx);
        std::vector<std::vector<double>> geoD_q;
        std::vector<Dense> geoE_q;
        for (int f = 0; f < op->NF; ++f) {
            geoD_q.push_back(grad_tandem(op->geo, fp[f], D));
            geoE_q.push_back(op->geo.eval(fp[f]));
        }
        const int DD = D * D;
        op->JInv.assign(static_cast<size_t>(op->E) * DD * op->Nq, 0.0);
        op->AbsDetJ.assign(static_cast<size_t>(op->E) * op->Nq, 0.0);
        op->Coords.assign(static_cast<size_t>(op->E) * D * op->Nq, 0.0);
        op->volume.assign(op->E, 0.0);
#pragma omp parallel for schedule(static)
        for (long el = 0; el < op->E; ++el) {
            std::vector<double> J(static_cast<size_t>(DD) * op->Nq);
            jacobian(*op, geo_nodes, el, geoD_Q, op->Nq, J.data());
            double vol = 0.0;
            for (int q = 0; q < op->Nq; ++q) {
                double det;
                inv_det(D, &J[static_cast<size_t>(DD) * q], &op->JInv[(static_cast<size_t>(el) * op->Nq + q) * DD], &det);
                op->AbsDetJ[static_cast<size_t>(el) * op->Nq + q] = std::fabs(det);
                vol += op->W[q] * std::fabs(det);
                const double* X = &geo_nodes[static_cast<size_t>(el) * op->Ngeo * D];
                for (int d = 0; d < D; ++d) {
                    double s = 0.0;
                    for (int n = 0; n < op->Ngeo; ++n) s += X[n * D + d] * geoE_Q(n, q);
                    op->Coords[(static_cast<size_t>(el) * op->Nq + q) * D + d] = s;
                }
            }
            op->volume[el] = vol;
        }
        auto refN = tdg::reference_normals(D);
        op->Normal.assign(static_cast<size_t>(op->F) * D * op->nq, 0.0);
        op->UnitNormal.assign(op->Normal.size(), 0.0);
        op->NormalLength.assign(static_cast<size_t>(op->F) * op->nq, 0.0);
        op->JInv0.assign(static_cast<size_t>(op->F) * DD * op->nq, 0.0);
        op->JInv1.assign(op->JInv0.size(), 0.0);
        op->FCoords.assign(static_cast<size_t>(op->F) * D * op->nq, 0.0);
        op->area.assign(op->F, 0.0);
#pragma omp parallel for schedule(static)
        for (long f = 0; f < op->F; ++f) {
            FacetInfo const& fi = op->fct[f];
            std::vector<double> J(static_cast<size_t>(DD) * op->nq);
            jacobian(*op, geo_nodes, fi.up[0], geoD_q[fi.localNo[0]], op->nq, J.data());
            double a = 0.0;
            for (int q = 0; q < op->nq; ++q) {
                double det;
                double* Ji = &op->JInv0[(static_cast<size_t>(f) * op->nq + q) * DD];
                inv_det(D, &J[static_cast<size_t>(DD) * q], Ji, &det);
                // n_i = |detJ| J^{-T}_{ij} N_j  with J^{-T}(i, j) = JInv(j, i)
                double nl2 = 0.0;
                for (int i = 0; i < D; ++i) {
                    double s = 0.0;
                    for (int j = 0; j < D; ++j) s += Ji[j + D * i] * refN[fi.localNo[0]][j];
                    op->Normal[(static_cast<size_t>(f) * op->nq + q) * D + i] = std::fabs(det) * s;
                    nl2 += (std::fabs(det) * s) * (std::fabs(det) * s);
                }
                double nl = std::sqrt(nl2);
                op->NormalLength[static_cast<size_t>(f) * op->nq + q] = nl;
                for (int i = 0; i < D; ++i)
                    op->UnitNormal[(static_cast<size_t>(f) * op->nq + q) * D + i] =
                        op->Normal[(static_cast<size_t>(f) * op->nq + q) * D + i] / nl;
                a += op->w[q] * nl;
                const double* X = &geo_nodes[static_cast<size_t>(fi.up[0]) * op->Ngeo * D];
                for (int d = 0; d < D; ++d) {
                    double s = 0.0;
                    for (int n = 0; n < op->Ngeo; ++n) s += X[n * D + d] * geoE_q[fi.localNo[0]](n, q);
                    op->FCoords[(static_cast<size_t>(f) * op->nq + q) * D + d] = s;
                }
            }
            op->area[f] = a;
            jacobian(*op, geo_nodes, fi.up[1], geoD_q[fi.localNo[1]], op->nq, J.data());
            for (int q = 0; q < op->nq; ++q) {
                double det;
                inv_det(D, &J[static_cast<size_t>(DD) * q], &op->JInv1[(static_cast<size_t>(f) * op->nq + q) * DD], &det);
            }
        }
        *out = op;
        return 0;
    } catch (std::exception const&) {
        return -1;
    }
}

void orc_destroy(orc_op* op) { delete op; }

void orc_volume_coords(orc_op const* op, double* out) {
    std::memcpy(out, op->Coords.data(), op->Coords.size() * sizeof(double));
}
void orc_facet_coords(orc_op const* op, double* out) {
    std::memcpy(out, op->FCoords.data(), op->FCoords.size() * sizeof(double));
}
void orc_facet_normals(orc_op const* op, double* out) {
    std::memcpy(out, op->Normal.data(), op->Normal.size() * sizeof(double));
}

int orc_set_material(orc_op* op, const double* c0_Q, const double* c1_Q) {
    const int D = op->D, Nq = op->Nq, nq = op->nq, nbf = op->Nbf, DD = D * D;
    op->matA.assign(static_cast<size_t>(op->E) * nbf, 0.0);
    op->matB.assign(static_cast<size_t>(op->E) * nbf, 0.0);
    op->vol0.assign(static_cast<size_t>(op->E) * Nq, 0.0);
    op->vol1.assign(static_cast<size_t>(op->E) * Nq, 0.0);
#pragma omp parallel for schedule(static)
    for (long el = 0; el < op->E; ++el) {
        const double* J = &op->AbsDetJ[static_cast<size_t>(el) * Nq];
        // project_K_lhs / project_material_lhs: matM(k, l) = matE(q, k) W J matE(q, l)
        Dense M(nbf, nbf);
        for (int k = 0; k < nbf; ++k)
            for (int l = 0; l < nbf; ++l) {
                double s = 0.0;
                for (int q = 0; q < Nq; ++q)
                    s += op->matE_Q[q + static_cast<size_t>(Nq) * k] * op->W[q] * J[q] * op->matE_Q[q + static_cast<size_t>(Nq) * l];
                M(k, l) = s;
            }
        for (int c = 0; c < (op->kind == kPoisson ? 1 : 2); ++c) {
            const double* cq = (c == 0 ? c0_Q : c1_Q) + static_cast<size_t>(el) * Nq;
            std::vector<double> b(nbf);
            for (int k = 0; k < nbf; ++k) {
                double s = 0.0;
                for (int q = 0; q < Nq; ++q) s += cq[q] * op->matE_Q[q + static_cast<size_t>(Nq) * k] * op->W[q] * J[q];
                b[k] = s;
            }
            tdg::solve_in_place(M, b.data());
            std::copy(b.begin(), b.end(), &(c == 0 ? op->matA : op->matB)[static_cast<size_t>(el) * nbf]);
        }
        // J_W_K_Q (Poisson) / precomputeVolume (Elasticity)
        for (int q = 0; q < Nq; ++q) {
            double a = 0.0, b = 0.0;
            for (int t = 0; t < nbf; ++t) {
                a += op->matE_Q[q + static_cast<size_t>(Nq) * t] * op->matA[static_cast<size_t>(el) * nbf + t];
                b += op->matE_Q[q + static_cast<size_t>(Nq) * t] * op->matB[static_cast<size_t>(el) * nbf + t];
            }
            op->vol0[static_cast<size_t>(el) * Nq + q] = J[q] * op->W[q] * a;
            op->vol1[static_cast<size_t>(el) * Nq + q] = b * op->W[q] * J[q];
        }
    }
    // facet precompute
    if (op->kind == kPoisson) {
        op->KG0.assign(static_cast<size_t>(op->F) * DD * nq, 0.0);
        op->KG1.assign(op->KG0.size(), 0.0);
    } else {
        op->lam0.assign(static_cast<size_t>(op->F) * nq, 0.0);
        op->mu0 = op->lam1 = op->mu1 = op->lam0;
    }
#pragma omp parallel for schedule(static)
    for (long f = 0; f < op->F; ++f) {
        FacetInfo const& fi = op->fct[f];
        for (int side = 0; side < 2; ++side) {
            long el = fi.up[side];
            auto const& mE = op->matE_q[fi.localNo[side]];
            for (int q = 0; q < nq; ++q) {
                double a = 0.0, b = 0.0;
                for (int t = 0; t < nbf; ++t) {
                    a += mE[q + static_cast<size_t>(nq) * t] * op->matA[static_cast<size_t>(el) * nbf + t];
                    b += mE[q + static_cast<size_t>(nq) * t] * op->matB[static_cast<size_t>(el) * nbf + t];
                }
                if (op->kind == kPoisson) {
                    const double* G = &(side == 0 ? op->JInv0 : op->JInv1)[(static_cast<size_t>(f) * nq + q) * DD];
                    double* out = &(side == 0 ? op->KG0 : op->KG1)[(static_cast<size_t>(f) * nq + q) * DD];
                    for (int c = 0; c < DD; ++c) out[c] = a * G[c];
                } else {
                    (side == 0 ? op->lam0 : op->lam1)[static_cast<size_t>(f) * nq + q] = a;
                    (side == 0 ? op->mu0 : op->mu1)[static_cast<size_t>(f) * nq + q] = b;
                }
            }
        }
    }
    // prepare_penalty
    op->penalty.assign(op->F, 0.0);
    const double cN1 = op->N * (op->N - 1.0 + D) / static_cast<double>(D);  // trace_constant(N - 1)
    for (long f = 0; f < op->F; ++f) {
        FacetInfo const& fi = op->fct[f];
        auto p = [&](int side) {
            long el = fi.up[side];
            double c0 = std::numeric_limits<double>::max(), c1 = std::numeric_limits<double>::lowest();
            for (int i = 0; i < nbf; ++i) {
                double a = op->matA[static_cast<size_t>(el) * nbf + i], b = op->matB[static_cast<size_t>(el) * nbf + i];
                if (op->kind == kPoisson) {
                    c0 = std::min(c0, a);
                    c1 = std::max(c1, a);
                } else {
                    c0 = std::min(c0, 2.0 * b);
                    c1 = std::max(c1, D * a + 2.0 * b);
                }
            }
            return (D + 1) * cN1 * (op->area[f] / op->volume[el]) * (c1 * c1 / c0);
        };
        op->penalty[f] = (fi.up[0] != fi.up[1]) ? (p(0) + p(1)) / 4.0 : p(0);
    }
    op->ready = true;
    op->pc.clear();
    return 0;
}

void orc_material_nodal(orc_op const* op, int c, double* out) {
    auto const& v = c == 0 ? op->matA : op->matB;
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void orc_penalty(orc_op const* op, double* out) { std::memcpy(out, op->penalty.data(), op->penalty.size() * sizeof(double)); }

}  // extern "C"

namespace {

// ---------------------------------------------------------------------------------------------
// element-centric apply (DGOperator::apply_ + LocalOperator::apply)
// ---------------------------------------------------------------------------------------------

void poisson_apply(orc_op const& op, long el, const double* x, double* y) {
    const int D = op.D, nbf = op.Nbf, Nq = op.Nq, nq = op.nq, DD = D * D;
    const double* U = x + static_cast<size_t>(el) * op.bs;
    double* Un = y + static_cast<size_t>(el) * op.bs;
    // apply_volume: Dx_Q(k, r, q) = Dxi_Q(k, e, q) G_Q(e, r, q);
    //               U_new(k) = J_W_K_Q(q) Dx_Q(k, r, q) Dx_Q(l, r, q) U(l)
    std::vector<double> Dx(static_cast<size_t>(nbf) * D * Nq);
    const double* G = &op.JInv[static_cast<size_t>(el) * Nq * DD];
    for (int q = 0; q < Nq; ++q)
        for (int r = 0; r < D; ++r)
            for (int k = 0; k < nbf; ++k) {
                double s = 0.0;
                for (int e = 0; e < D; ++e) s += op.Dxi_Q[idx3(k, e, q, nbf, D)] * G[q * DD + e + D * r];
                Dx[idx3(k, r, q, nbf, D)] = s;
            }
    for (int k = 0; k < nbf; ++k) Un[k] = 0.0;
    for (int q = 0; q < Nq; ++q) {
        const double jwk = op.vol0[static_cast<size_t>(el) * Nq + q];
        for (int r = 0; r < D; ++r) {
            double g = 0.0;
            for (int l = 0; l < nbf; ++l) g += Dx[idx3(l, r, q, nbf, D)] * U[l];
            for (int k = 0; k < nbf; ++k) Un[k] += jwk * Dx[idx3(k, r, q, nbf, D)] * g;
        }
    }
    std::vector<double> n_q(static_cast<size_t>(D) * nq), nu_q(static_cast<size_t>(D) * nq);
    std::vector<double> uh(nq), sig(static_cast<size_t>(D) * nq);
    for (int f = 0; f < op.NF; ++f) {
        SideInfo const& si = op.sides[el * op.NF + f];
        const bool skel = el != si.lid;
        const bool fd = si.bc == BC_Fault || si.bc == BC_Dirichlet;
        const long fc = si.fctNo;
        const double* KG0 = &op.KG0[static_cast<size_t>(fc) * nq * DD];
        const double* KG1 = &op.KG1[static_cast<size_t>(fc) * nq * DD];
        const double sgn = (skel && si.side == 1) ? -1.0 : 1.0;
        if (skel && si.side == 1) std::swap(KG0, KG1);
        for (int q = 0; q < nq; ++q)
            for (int d = 0; d < D; ++d) {
                n_q[d + D * q] = sgn * op.Normal[(static_cast<size_t>(fc) * nq + q) * D + d];
                nu_q[d + D * q] = sgn * op.UnitNormal[(static_cast<size_t>(fc) * nq + q) * D + d];
            }
        const double c00 = -op.penalty[fc];
        auto const& E0 = op.E_q[f];
        auto const& D0 = op.Dxi_q[f];
        if (si.bc == BC_None || (skel && fd)) {
            auto const& E1 = op.E_q[si.localNo];
            auto const& D1 = op.Dxi_q[si.localNo];
            const double* Ue = x + static_cast<size_t>(si.lid) * op.bs;
            for (int q = 0; q < nq; ++q) {
                double e0 = 0.0, e1 = 0.0;
                for (int l = 0; l < nbf; ++l) {
                    e0 += E0[l + static_cast<size_t>(nbf) * q] * U[l];
                    e1 += E1[l + static_cast<size_t>(nbf) * q] * Ue[l];
                }
                uh[q] = 0.5 * (-e0 + e1);  // flux_u_skeleton
                for (int p = 0; p < D; ++p) {
                    double s = 0.0;
                    for (int e = 0; e < D; ++e) {
                        double g0 = 0.0, g1 = 0.0;
                        for (int l = 0; l < nbf; ++l) {
                            g0 += D0[idx3(l, e, q, nbf, D)] * U[l];
                            g1 += D1[idx3(l, e, q, nbf, D)] * Ue[l];
                        }
                        s += KG0[q * DD + e + D * p] * g0 + KG1[q * DD + e + D * p] * g1;
                    }
                    sig[p + D * q] = 0.5 * s + c00 * (e0 - e1) * nu_q[p + D * q];  // flux_sigma_skeleton
                }
            }
        } else if (fd) {
            for (int q = 0; q < nq; ++q) {
                double e0 = 0.0;
                for (int l = 0; l < nbf; ++l) e0 += E0[l + static_cast<size_t>(nbf) * q] * U[l];
                uh[q] = -e0;  // flux_u_boundary
                for (int p = 0; p < D; ++p) {
                    double s = 0.0;
                    for (int e = 0; e < D; ++e) {
                        double g0 = 0.0;
                        for (int l = 0; l < nbf; ++l) g0 += D0[idx3(l, e, q, nbf, D)] * U[l];
                        s += KG0[q * DD + e + D * p] * g0;
                    }
                    sig[p + D * q] = s + c00 * e0 * nu_q[p + D * q];  // flux_sigma_boundary
                }
            }
        } else {
            continue;
        }
        // apply_facet: U_new(k) += w(q) n(r, q) (u_hat(q) K_G_q0(e, r, q) Dxi_q(k, e, q) - E_q(k, q) sigma_hat(r, q))
        for (int q = 0; q < nq; ++q)
            for (int r = 0; r < D; ++r) {
                const double wn = op.w[q] * n_q[r + D * q];
                for (int k = 0; k < nbf; ++k) {
                    double kd = 0.0;
                    for (int e = 0; e < D; ++e) kd += KG0[q * DD + e + D * r] * D0[idx3(k, e, q, nbf, D)];
                    Un[k] += wn * (uh[q] * kd - E0[k + static_cast<size_t>(nbf) * q] * sig[r + D * q]);
                }
            }
    }
}

void elasticity_apply(orc_op const& op, long el, const double* x, double* y) {
    const int D = op.D, nbf = op.Nbf, Nq = op.Nq, nq = op.nq, DD = D * D;
    const double* U = x + static_cast<size_t>(el) * op.bs;  // U(l, r) at l + nbf r
    double* Un = y + static_cast<size_t>(el) * op.bs;
    const double* G = &op.JInv[static_cast<size_t>(el) * Nq * DD];  // G(e, j, q)
    for (int i = 0; i < op.bs; ++i) Un[i] = 0.0;
    // apply_volume: Ju_Q(q, s, r) = G_Q_T(s, e, q) Dxi_Q_120(e, q, l) U(l, r)  [G_T(s, e) = G(e, s)]
    //   Unew(k, u) = Dxi_Q(k, e, q) G(e, j, q) (lamWJ delta_uj delta_rs Ju(q, r, s) + muWJ (Ju(q, u, j) + Ju(q, j, u)))
    for (int q = 0; q < Nq; ++q) {
        double Ju[3][3];  // Ju[s][r]
        for (int s = 0; s < D; ++s)
            for (int r = 0; r < D; ++r) {
                double acc = 0.0;
                for (int e = 0; e < D; ++e) {
                    double g = 0.0;
                    for (int l = 0; l < nbf; ++l) g += op.Dxi_Q[idx3(l, e, q, nbf, D)] * U[l + nbf * r];
                    acc += G[q * DD + e + D * s] * g;
                }
                Ju[s][r] = acc;
            }
        const double lam = op.vol0[static_cast<size_t>(el) * Nq + q], mu = op.vol1[static_cast<size_t>(el) * Nq + q];
        double tr = 0.0;
        for (int r = 0; r < D; ++r) tr += Ju[r][r];
        for (int u = 0; u < D; ++u)
            for (int j = 0; j < D; ++j) {
                const double sig = (u == j ? lam * tr : 0.0) + mu * (Ju[u][j] + Ju[j][u]);
                for (int e = 0; e < D; ++e) {
                    const double gs = G[q * DD + e + D * j] * sig;
                    for (int k = 0; k < nbf; ++k) Un[k + nbf * u] += op.Dxi_Q[idx3(k, e, q, nbf, D)] * gs;
                }
            }
    }
    std::vector<double> uhm(static_cast<size_t>(nq) * D), sigh(static_cast<size_t>(DD) * nq);
    for (int f = 0; f < op.NF; ++f) {
        SideInfo const& si = op.sides[el * op.NF + f];
        const bool skel = el != si.lid;
        const bool fd = si.bc == BC_Fault || si.bc == BC_Dirichlet;
        const long fc = si.fctNo;
        const double* l0 = &op.lam0[static_cast<size_t>(fc) * nq];
        const double* l1 = &op.lam1[static_cast<size_t>(fc) * nq];
        const double* m0 = &op.mu0[static_cast<size_t>(fc) * nq];
        const double* m1 = &op.mu1[static_cast<size_t>(fc) * nq];
        const double* G0 = &op.JInv0[static_cast<size_t>(fc) * nq * DD];
        const double* G1 = &op.JInv1[static_cast<size_t>(fc) * nq * DD];
        const double sgn = (skel && si.side == 1) ? -1.0 : 1.0;
        if (skel && si.side == 1) {
            std::swap(l0, l1);
            std::swap(m0, m1);
            std::swap(G0, G1);
        }
        auto nrm = [&](int d, int q) { return sgn * op.Normal[(static_cast<size_t>(fc) * nq + q) * D + d]; };
        auto nun = [&](int d, int q) { return sgn * op.UnitNormal[(static_cast<size_t>(fc) * nq + q) * D + d]; };
        const double c00 = -op.penalty[fc];
        auto const& E0 = op.E_q[f];
        auto const& D0 = op.Dxi_q[f];
        // Ju_q(q, r, s) = G_q_T(s, e, q) Dxi_q_120(e, q, l) U(l, r) = G(e, s) dU_r/dxi_e
        auto ju = [&](const double* Gs, std::vector<double> const& Dq, const double* V, int q, double J[3][3]) {
            for (int r = 0; r < D; ++r)
                for (int s = 0; s < D; ++s) {
                    double acc = 0.0;
                    for (int e = 0; e < D; ++e) {
                        double g = 0.0;
                        for (int l = 0; l < nbf; ++l) g += Dq[idx3(l, e, q, nbf, D)] * V[l + nbf * r];
                        acc += Gs[q * DD + e + D * s] * g;
                    }
                    J[r][s] = acc;  // J[r][s] = Ju_q(q, r, s)
                }
        };
        // constitutive_q(x)(i, j, q) = lam delta_ij delta_rs Ju(q, r, s) + mu (Ju(q, i, j) + Ju(q, j, i))
        auto constitutive = [&](double lam, double mu, double J[3][3], double S[3][3]) {
            double tr = 0.0;
            for (int r = 0; r < D; ++r) tr += J[r][r];
            for (int i = 0; i < D; ++i)
                for (int j = 0; j < D; ++j) S[i][j] = (i == j ? lam * tr : 0.0) + mu * (J[i][j] + J[j][i]);
        };
        if (si.bc == BC_None || (skel && fd)) {
            auto const& E1 = op.E_q[si.localNo];
            auto const& D1 = op.Dxi_q[si.localNo];
            const double* Ue = x + static_cast<size_t>(si.lid) * op.bs;
            for (int q = 0; q < nq; ++q) {
                double J0[3][3], J1[3][3], S0[3][3], S1[3][3];
                ju(G0, D0, U, q, J0);
                ju(G1, D1, Ue, q, J1);
                constitutive(l0[q], m0[q], J0, S0);
                constitutive(l1[q], m1[q], J1, S1);
                for (int i = 0; i < D; ++i) {
                    double e0 = 0.0, e1 = 0.0;
                    for (int l = 0; l < nbf; ++l) {
                        e0 += E0[l + static_cast<size_t>(nbf) * q] * U[l + nbf * i];
                        e1 += E1[l + static_cast<size_t>(nbf) * q] * Ue[l + nbf * i];
                    }
                    uhm[q + static_cast<size_t>(nq) * i] = 0.5 * (-e0 + e1);
                    for (int j = 0; j < D; ++j)
                        sigh[i + D * (j + D * q)] = 0.5 * (S0[i][j] + S1[i][j]) + c00 * (e0 - e1) * nun(j, q);
                }
            }
        } else if (fd) {
            for (int q = 0; q < nq; ++q) {
                double J0[3][3], S0[3][3];
                ju(G0, D0, U, q, J0);
                constitutive(l0[q], m0[q], J0, S0);
                for (int i = 0; i < D; ++i) {
                    double e0 = 0.0;
                    for (int l = 0; l < nbf; ++l) e0 += E0[l + static_cast<size_t>(nbf) * q] * U[l + nbf * i];
                    uhm[q + static_cast<size_t>(nq) * i] = -e0;
                    for (int j = 0; j < D; ++j) sigh[i + D * (j + D * q)] = S0[i][j] + c00 * e0 * nun(j, q);
                }
            }
        } else {
            continue;
        }
        // apply_facet: Unew(k, u) += w G_q_T0(j, e, q) Dxi_q(k, e, q) (lam0 delta_uj uhm(q, r) n(r, q)
        //      + mu0 (uhm(q, u) n(j, q) + uhm(q, j) n(u, q))) + w (-E_q(k, q)) n(j, q) sigma_hat(u, j, q)
        for (int q = 0; q < nq; ++q) {
            double un = 0.0;
            for (int r = 0; r < D; ++r) un += uhm[q + static_cast<size_t>(nq) * r] * nrm(r, q);
            for (int u = 0; u < D; ++u)
                for (int j = 0; j < D; ++j) {
                    const double X = (u == j ? l0[q] * un : 0.0) +
                                     m0[q] * (uhm[q + static_cast<size_t>(nq) * u] * nrm(j, q) +
                                              uhm[q + static_cast<size_t>(nq) * j] * nrm(u, q));
                    const double sn = nrm(j, q) * sigh[u + D * (j + D * q)];
                    for (int k = 0; k < nbf; ++k) {
                        double gd = 0.0;
                        for (int e = 0; e < D; ++e) gd += G0[q * DD + e + D * j] * D0[idx3(k, e, q, nbf, D)];
                        Un[k + nbf * u] += op.w[q] * (gd * X - E0[k + static_cast<size_t>(nbf) * q] * sn);
                    }
                }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// assemble: diagonal blocks, column-major [col * bs + row]
// ---------------------------------------------------------------------------------------------

void assemble_block(orc_op const& op, long el, double* A) {
    const int D = op.D, nbf = op.Nbf, Nq = op.Nq, nq = op.nq, DD = D * D, bs = op.bs;
    std::fill(A, A + static_cast<size_t>(bs) * bs, 0.0);
    const double* G = &op.JInv[static_cast<size_t>(el) * Nq * DD];
    std::vector<double> Dx(static_cast<size_t>(nbf) * D * Nq);  // Dx_Q(k, i, q) = G(e, i) Dxi(k, e)
    for (int q = 0; q < Nq; ++q)
        for (int i = 0; i < D; ++i)
            for (int k = 0; k < nbf; ++k) {
                double s = 0.0;
                for (int e = 0; e < D; ++e) s += G[q * DD + e + D * i] * op.Dxi_Q[idx3(k, e, q, nbf, D)];
                Dx[idx3(k, i, q, nbf, D)] = s;
            }
    auto at = [&](int k, int p, int l, int u) -> double& { return A[(k + nbf * p) + static_cast<size_t>(bs) * (l + nbf * u)]; };
    for (int q = 0; q < Nq; ++q) {
        const double c0 = op.vol0[static_cast<size_t>(el) * Nq + q], c1 = op.vol1[static_cast<size_t>(el) * Nq + q];
        for (int k = 0; k < nbf; ++k)
            for (int l = 0; l < nbf; ++l) {
                double kl = 0.0;
                for (int i = 0; i < D; ++i) kl += Dx[idx3(k, i, q, nbf, D)] * Dx[idx3(l, i, q, nbf, D)];
                if (op.kind == kPoisson) {
                    at(k, 0, l, 0) += c0 * kl;  // assembleVolume: J W K Dx Dx
                } else {
                    for (int p = 0; p < D; ++p)
                        for (int u = 0; u < D; ++u)
                            at(k, p, l, u) += c0 * Dx[idx3(l, u, q, nbf, D)] * Dx[idx3(k, p, q, nbf, D)] +
                                              c1 * ((p == u ? kl : 0.0) + Dx[idx3(k, u, q, nbf, D)] * Dx[idx3(l, p, q, nbf, D)]);
                }
            }
    }
    for (int f = 0; f < op.NF; ++f) {
        SideInfo const& si = op.sides[el * op.NF + f];
        const bool skel = el != si.lid;
        const long fc = si.fctNo;
        FacetInfo const& fi = op.fct[fc];
        if (!skel && !(fi.bc == BC_Fault || fi.bc == BC_Dirichlet)) continue;  // assemble_boundary: Natural -> none
        const int x = skel ? si.side : 0;  // which diagonal block a(x, x) of the facet this element gets
        // constants of assembleSurface: interior c0x = (-1/2, +1/2), c1x = (eps/2, -eps/2), c20 = penalty;
        // boundary c00 = -1, c10 = eps, c20 = penalty; eps = -1
        double c0, c1;
        if (skel) {
            c0 = (x == 0) ? -0.5 : 0.5;
            c1 = (x == 0) ? -0.5 : 0.5;
        } else {
            c0 = -1.0;
            c1 = -1.0;
        }
        const double c2 = op.penalty[fc];
        auto const& Eq = op.E_q[fi.localNo[x]];
        auto const& Dq = op.Dxi_q[fi.localNo[x]];
        const double* Gx = &(x == 0 ? op.JInv0 : op.JInv1)[static_cast<size_t>(fc) * nq * DD];
        std::vector<double> Dxq(static_cast<size_t>(nbf) * D * nq);
        for (int q = 0; q < nq; ++q)
            for (int i = 0; i < D; ++i)
                for (int k = 0; k < nbf; ++k) {
                    double s = 0.0;
                    for (int e = 0; e < D; ++e) s += Gx[q * DD + e + D * i] * Dq[idx3(k, e, q, nbf, D)];
                    Dxq[idx3(k, i, q, nbf, D)] = s;
                }
        for (int q = 0; q < nq; ++q) {
            const double wq = op.w[q], nl = op.NormalLength[static_cast<size_t>(fc) * nq + q];
            const double* n = &op.Normal[(static_cast<size_t>(fc) * nq + q) * D];
            if (op.kind == kPoisson) {
                // K_Dx_q(k, i, q) = K_q Dx_q; lift_ip L_q(l, q) = E_q(l, q) nl_q
                double Kq = 0.0;
                for (int t = 0; t < nbf; ++t)
                    Kq += op.matE_q[fi.localNo[x]][q + static_cast<size_t>(nq) * t] * op.matA[static_cast<size_t>(fi.up[x]) * nbf + t];
                for (int k = 0; k < nbf; ++k)
                    for (int l = 0; l < nbf; ++l) {
                        double dk = 0.0, dl = 0.0;
                        for (int i = 0; i < D; ++i) {
                            dk += Kq * Dxq[idx3(k, i, q, nbf, D)] * n[i];
                            dl += Kq * Dxq[idx3(l, i, q, nbf, D)] * n[i];
                        }
                        const double ek = Eq[k + static_cast<size_t>(nbf) * q], elv = Eq[l + static_cast<size_t>(nbf) * q];
                        at(k, 0, l, 0) += c0 * wq * dk * elv + c1 * wq * dl * ek + c2 * wq * ek * elv * nl;
                    }
            } else {
                const double lam = (x == 0 ? op.lam0 : op.lam1)[static_cast<size_t>(fc) * nq + q];
                const double mu = (x == 0 ? op.mu0 : op.mu1)[static_cast<size_t>(fc) * nq + q];
                // traction_op_q(k, p, u, q) = lam Dx(k, p) n(u) + mu (n(j) Dx(k, j) delta_pu + Dx(k, u) n(p))
                auto T = [&](int k, int p, int u) {
                    double dn = 0.0;
                    for (int j = 0; j < D; ++j) dn += n[j] * Dxq[idx3(k, j, q, nbf, D)];
                    return lam * Dxq[idx3(k, p, q, nbf, D)] * n[u] + mu * ((p == u ? dn : 0.0) + Dxq[idx3(k, u, q, nbf, D)] * n[p]);
                };
                for (int k = 0; k < nbf; ++k)
                    for (int p = 0; p < D; ++p)
                        for (int l = 0; l < nbf; ++l)
                            for (int u = 0; u < D; ++u) {
                                const double ek = Eq[k + static_cast<size_t>(nbf) * q], elv = Eq[l + static_cast<size_t>(nbf) * q];
                                // a(x, x)(k, p, l, u) = c0 E(k) w T(l, u, p) + c1 E(l) w T(k, p, u) + c2 w E(k) E(l) delta_pu nl
                                at(k, p, l, u) += c0 * ek * wq * T(l, u, p) + c1 * elv * wq * T(k, p, u) +
                                                  (p == u ? c2 * wq * ek * elv * nl : 0.0);
                            }
            }
        }
    }
}

}  // namespace

extern "C" {

void orc_apply(orc_op const* op, const double* x, double* y) {
#pragma omp parallel for schedule(dynamic, 64)
    for (long el = 0; el < op->E; ++el) {
        if (op->kind == kPoisson)
            poisson_apply(*op, el, x, y);
        else
            elasticity_apply(*op, el, x, y);
    }
}

// Applies the operator to the element range [e0, e1) only (bounded CPU timing samples).
void orc_apply_range(orc_op const* op, long e0, long e1, const double* x, double* y) {
#pragma omp parallel for schedule(dynamic, 64)
    for (long el = e0; el < e1; ++el) {
        if (op->kind == kPoisson)
            poisson_apply(*op, el, x, y);
        else
            elasticity_apply(*op, el, x, y);
    }
}

void orc_assemble_diag(orc_op const* op, double* blocks) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long el = 0; el < op->E; ++el) assemble_block(*op, el, blocks + static_cast<size_t>(el) * op->bs * op->bs);
}

// rhs (DGOperator::rhs): force_Q [E][Q][Nq], bc_q [F][Q][nq]
void orc_rhs(orc_op const* op, const double* force_Q, const double* bc_q, double* b) {
    const int D = op->D, nbf = op->Nbf, Nq = op->Nq, nq = op->nq, DD = D * D, Q = op->Q;
    std::fill(b, b + static_cast<size_t>(op->E) * op->bs, 0.0);
    if (force_Q) {
        for (long el = 0; el < op->E; ++el)
            for (int p = 0; p < Q; ++p)
                for (int k = 0; k < nbf; ++k) {
                    double s = 0.0;
                    for (int q = 0; q < Nq; ++q)
                        s += op->AbsDetJ[static_cast<size_t>(el) * Nq + q] * op->W[q] * op->E_Q[k + static_cast<size_t>(nbf) * q] *
                             force_Q[(static_cast<size_t>(el) * Q + p) * Nq + q];
                    b[static_cast<size_t>(el) * op->bs + k + nbf * p] += s;
                }
    }
    if (!bc_q) return;
    for (long fc = 0; fc < op->F; ++fc) {
        FacetInfo const& fi = op->fct[fc];
        if (fi.bc != BC_Fault && fi.bc != BC_Dirichlet) continue;
        const bool boundary = fi.up[0] == fi.up[1];
        std::vector<double> f_q(static_cast<size_t>(Q) * nq);
        for (int i = 0; i < Q * nq; ++i) {
            f_q[i] = bc_q[static_cast<size_t>(fc) * Q * nq + i];
            if (boundary && fi.bc == BC_Fault) f_q[i] *= 0.5;
        }
        for (int side = 0; side < (boundary ? 1 : 2); ++side) {
            const double c10 = boundary ? -1.0 : -0.5;
            const double c20 = side == 0 ? op->penalty[fc] : -op->penalty[fc];
            const long el = fi.up[side];
            auto const& Eq = op->E_q[fi.localNo[side]];
            auto const& Dq = op->Dxi_q[fi.localNo[side]];
            const double* Gs = &(side == 0 ? op->JInv0 : op->JInv1)[static_cast<size_t>(fc) * nq * DD];
            double* bb = b + static_cast<size_t>(el) * op->bs;
            for (int q = 0; q < nq; ++q) {
                const double* n = &op->Normal[(static_cast<size_t>(fc) * nq + q) * D];
                const double nl = op->NormalLength[static_cast<size_t>(fc) * nq + q];
                const double wq = op->w[q];
                for (int k = 0; k < nbf; ++k) {
                    double Dx[3];
                    for (int i = 0; i < D; ++i) {
                        double s = 0.0;
                        for (int e = 0; e < D; ++e) s += Gs[q * DD + e + D * i] * Dq[idx3(k, e, q, nbf, D)];
                        Dx[i] = s;
                    }
                    const double ek = Eq[k + static_cast<size_t>(nbf) * q];
                    if (op->kind == kPoisson) {
                        double Kq = 0.0;
                        for (int t = 0; t < nbf; ++t)
                            Kq += op->matE_q[fi.localNo[side]][q + static_cast<size_t>(nq) * t] * op->matA[static_cast<size_t>(el) * nbf + t];
                        double dn = 0.0;
                        for (int i = 0; i < D; ++i) dn += Kq * Dx[i] * n[i];
                        // rhsFacet: c10 w K_Dx n f + c20 w E f_lifted, f_lifted = nl f (rhs_lift_ip)
                        bb[k] += c10 * wq * dn * f_q[q] + c20 * wq * ek * nl * f_q[q];
                    } else {
                        const double lam = (side == 0 ? op->lam0 : op->lam1)[static_cast<size_t>(fc) * nq + q];
                        const double mu = (side == 0 ? op->mu0 : op->mu1)[static_cast<size_t>(fc) * nq + q];
                        double fn = 0.0, dxn = 0.0, dxf = 0.0;
                        for (int i = 0; i < D; ++i) {
                            fn += f_q[q + static_cast<size_t>(nq) * i] * n[i];
                            dxn += Dx[i] * n[i];
                            dxf += Dx[i] * f_q[q + static_cast<size_t>(nq) * i];
                        }
                        for (int p = 0; p < D; ++p) {
                            // tractionTest(0, f)(k, p) = lam Dx(k, p) f.n + mu (Dx.n f_p + Dx.f n_p)
                            const double tt = lam * Dx[p] * fn + mu * (dxn * f_q[q + static_cast<size_t>(nq) * p] + dxf * n[p]);
                            bb[k + nbf * p] += c10 * wq * tt + c20 * wq * ek * nl * f_q[q + static_cast<size_t>(nq) * p];
                        }
                    }
                }
            }
        }
    }
}

// Block-Jacobi preconditioned CG (FP64) on the unpreconditioned residual: stops when the true
// relative residual ||b - A x|| / ||b|| <= rtol.  Returns 0 on convergence.
// 1/rho at the volume points, projected onto the nodal material space (project_material_lhs /
// project_material_rhs with rhoInv_Q = 1 / rho_Q, Elasticity.cpp:104-175)
int orc_set_density(orc_op* op, const double* rho_Q) {
    const int Nq = op->Nq, nbf = op->Nbf;
    op->rhoInv.assign(static_cast<size_t>(op->E) * nbf, 0.0);
#pragma omp parallel for schedule(static)
    for (long el = 0; el < op->E; ++el) {
        const double* J = &op->AbsDetJ[static_cast<size_t>(el) * Nq];
        Dense M(nbf, nbf);
        for (int k = 0; k < nbf; ++k)
            for (int l = 0; l < nbf; ++l) {
                double s = 0.0;
                for (int q = 0; q < Nq; ++q)
                    s += op->matE_Q[q + static_cast<size_t>(Nq) * k] * op->W[q] * J[q] * op->matE_Q[q + static_cast<size_t>(Nq) * l];
                M(k, l) = s;
            }
        std::vector<double> b(nbf);
        for (int k = 0; k < nbf; ++k) {
            double s = 0.0;
            for (int q = 0; q < Nq; ++q)
                s += (1.0 / rho_Q[static_cast<size_t>(el) * Nq + q]) * op->matE_Q[q + static_cast<size_t>(Nq) * k] * op->W[q] * J[q];
            b[k] = s;
        }
        tdg::solve_in_place(M, b.data());
        std::copy(b.begin(), b.end(), &op->rhoInv[static_cast<size_t>(el) * nbf]);
    }
    return 0;
}

// Unew(k, p) = MinvRef(k, r) Jinv_Q(q) E_Q(r, q) E_Q(s, q) MinvRef(s, l) U(l, p) with
// Jinv_Q(q) = -rhoInv(q) W(q) / |J|(q) (apply_inverse_mass of Elasticity::wave_rhs)
void orc_apply_inverse_mass(orc_op const* op, const double* x, double* y) {
    const int Nq = op->Nq, nbf = op->Nbf, Q = op->Q;
    Dense Minv = tdg::invert(op->space.mass_matrix());
#pragma omp parallel for schedule(static)
    for (long el = 0; el < op->E; ++el) {
        const double* U = x + static_cast<size_t>(el) * op->bs;
        double* Y = y + static_cast<size_t>(el) * op->bs;
        std::vector<double> a(static_cast<size_t>(nbf) * Q, 0.0), b(static_cast<size_t>(nbf) * Q, 0.0);
        for (int p = 0; p < Q; ++p)
            for (int s = 0; s < nbf; ++s) {
                double t = 0.0;
                for (int l = 0; l < nbf; ++l) t += Minv(s, l) * U[l + nbf * p];
                a[s + nbf * p] = t;
            }
        for (int q = 0; q < Nq; ++q) {
            double ri = 1.0;
            if (!op->rhoInv.empty()) {
                ri = 0.0;
                for (int t = 0; t < nbf; ++t)
                    ri += op->matE_Q[q + static_cast<size_t>(Nq) * t] * op->rhoInv[static_cast<size_t>(el) * nbf + t];
            }
            const double jq = -ri * op->W[q] / op->AbsDetJ[static_cast<size_t>(el) * Nq + q];
            for (int p = 0; p < Q; ++p) {
                double v = 0.0;
                for (int s = 0; s < nbf; ++s) v += op->E_Q[s + static_cast<size_t>(nbf) * q] * a[s + nbf * p];
                v *= jq;
                for (int r = 0; r < nbf; ++r) b[r + nbf * p] += op->E_Q[r + static_cast<size_t>(nbf) * q] * v;
            }
        }
        for (int p = 0; p < Q; ++p)
            for (int k = 0; k < nbf; ++k) {
                double t = 0.0;
                for (int r = 0; r < nbf; ++r) t += Minv(k, r) * b[r + nbf * p];
                Y[k + nbf * p] = t;
            }
    }
}

int orc_cg(orc_op* op, const double* b, double* x, double rtol, int maxit, int* iters, double* relres) {
    const long n = op->E * op->bs;
    const int bs = op->bs;
    if (op->pc.empty()) {
        op->pc.assign(static_cast<size_t>(op->E) * bs * bs, 0.0);
        orc_assemble_diag(op, op->pc.data());
#pragma omp parallel for schedule(dynamic, 16)
        for (long el = 0; el < op->E; ++el) {
            Dense m(bs, bs);
            double* A = &op->pc[static_cast<size_t>(el) * bs * bs];
            for (int r = 0; r < bs; ++r)
                for (int c = 0; c < bs; ++c) m(r, c) = A[r + static_cast<size_t>(bs) * c];
            Dense inv = tdg::invert(m);
            for (int r = 0; r < bs; ++r)
                for (int c = 0; c < bs; ++c) A[r + static_cast<size_t>(bs) * c] = inv(r, c);
        }
    }
    std::vector<double> r(n), z(n), p(n), q(n);
    auto pcapply = [&](const double* in, double* out) {
#pragma omp parallel for schedule(static)
        for (long el = 0; el < op->E; ++el) {
            const double* M = &op->pc[static_cast<size_t>(el) * bs * bs];
            for (int row = 0; row < bs; ++row) {
                double s = 0.0;
                for (int c = 0; c < bs; ++c) s += M[row + static_cast<size_t>(bs) * c] * in[el * bs + c];
                out[el * bs + row] = s;
            }
        }
    };
    auto dot = [&](const double* a, const double* c) {
        double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (long i = 0; i < n; ++i) s += a[i] * c[i];
        return s;
    };
    const double bn = std::sqrt(dot(b, b));
    int it = 0;
    double rel = 0.0;
    for (int restart = 0; restart < 4; ++restart) {
        orc_apply(op, x, q.data());
        for (long i = 0; i < n; ++i) r[i] = b[i] - q[i];
        rel = bn > 0 ? std::sqrt(dot(r.data(), r.data())) / bn : 0.0;
        if (rel <= rtol || it >= maxit) break;
        pcapply(r.data(), z.data());
        p = z;
        double rz = dot(r.data(), z.data());
        while (it < maxit) {
            orc_apply(op, p.data(), q.data());
            const double alpha = rz / dot(p.data(), q.data());
#pragma omp parallel for schedule(static)
            for (long i = 0; i < n; ++i) {
                x[i] += alpha * p[i];
                r[i] -= alpha * q[i];
            }
            ++it;
            const double rr = std::sqrt(dot(r.data(), r.data()));
            if (!std::isfinite(rr)) return -4;
            if (rr <= rtol * bn) break;
            pcapply(r.data(), z.data());
            const double rz2 = dot(r.data(), z.data());
            const double beta = rz2 / rz;
            rz = rz2;
#pragma omp parallel for schedule(static)
            for (long i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        }
    }
    *iters = it;
    *relres = rel;
    return rel <= rtol ? 0 : -4;
}

// Error<D>::L2 with the operator's volume rule: ref_Q [E][Nq][Q] reference solution at the
// volume points.
double orc_error_L2(orc_op const* op, const double* x, const double* ref_Q) {
    double err = 0.0;
    const int nbf = op->Nbf, Nq = op->Nq, Q = op->Q;
#pragma omp parallel for reduction(+ : err) schedule(static)
    for (long el = 0; el < op->E; ++el)
        for (int j = 0; j < Q; ++j)
            for (int q = 0; q < Nq; ++q) {
                double v = 0.0;
                for (int k = 0; k < nbf; ++k) v += op->E_Q[k + static_cast<size_t>(nbf) * q] * x[el * op->bs + k + nbf * j];
                const double e = ref_Q[(static_cast<size_t>(el) * Nq + q) * Q + j] - v;
                err += op->W[q] * op->AbsDetJ[static_cast<size_t>(el) * Nq + q] * e * e;
            }
    return std::sqrt(err);
}

// Error<D>::H1_semi: refgrad_Q [E][Nq][Q][D] = d u_j / d x_d at the volume points.
double orc_error_H1_semi(orc_op const* op, const double* x, const double* refgrad_Q) {
    double err = 0.0;
    const int D = op->D, nbf = op->Nbf, Nq = op->Nq, Q = op->Q, DD = D * D;
#pragma omp parallel for reduction(+ : err) schedule(static)
    for (long el = 0; el < op->E; ++el)
        for (int q = 0; q < Nq; ++q) {
            const double* G = &op->JInv[(static_cast<size_t>(el) * Nq + q) * DD];
            for (int j = 0; j < Q; ++j)
                for (int d = 0; d < D; ++d) {
                    double v = 0.0;
                    for (int k = 0; k < nbf; ++k) {
                        double dx = 0.0;
                        for (int e = 0; e < D; ++e) dx += G[e + D * d] * op->Dxi_Q[idx3(k, e, q, nbf, D)];
                        v += dx * x[el * op->bs + k + nbf * j];
                    }
                    const double e = refgrad_Q[((static_cast<size_t>(el) * Nq + q) * Q + j) * D + d] - v;
                    err += op->W[q] * op->AbsDetJ[static_cast<size_t>(el) * Nq + q] * e * e;
                }
        }
    return std::sqrt(err);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Fault adapter (Poisson): AdapterBase::prepare (app/localoperator/AdapterBase.cpp:44-99),
// Adapter<Poisson>::slip / traction (app/localoperator/PoissonAdapter.cpp:22-55),
// Poisson::traction_skeleton / traction_boundary (Poisson.cpp:678-723, kernels grad_u /
// grad_u_bnd of app/kernels/poisson.py:146-152, evaluate_slip / evaluate_traction of
// poisson_adapter.py:13-23).
// ---------------------------------------------------------------------------------------------

extern "C" {

// slip_q on the fault facets: bc_q [F][nq] (zero elsewhere).  slip [nfault][nbf]; e_q [nbf][nq]
// is the fault basis at the facet points (passed in; computed by the caller from tandem's nodal
// warp & blend fault space).
void orc_fault_slip_q(orc_op const* op, long nfault, const long* facets, const double* ref_normal, const double* e_q,
                      int nbf, const double* slip, double* bc_q) {
    const int D = op->D, nq = op->nq;
    std::fill(bc_q, bc_q + static_cast<size_t>(op->F) * nq, 0.0);
    for (long i = 0; i < nfault; ++i) {
        const long fc = facets[i];
        for (int q = 0; q < nq; ++q) {
            double dot = 0.0;
            for (int d = 0; d < D; ++d) dot += ref_normal[d] * op->Normal[(static_cast<size_t>(fc) * nq + q) * D + d];
            double s = 0.0;
            for (int p = 0; p < nbf; ++p) s += e_q[p * nq + q] * slip[i * nbf + p];
            bc_q[static_cast<size_t>(fc) * nq + q] = dot < 0 ? -s : s;
        }
    }
}

// traction [nfault][nbf] of displacement u and slip [nfault][nbf].
void orc_fault_traction(orc_op const* op, long nfault, const long* facets, const double* ref_normal, const double* e_q,
                        int nbf, const double* u, const double* slip, double* traction) {
    const int D = op->D, nq = op->nq, nbfe = op->Nbf, DD = D * D;
    for (long i = 0; i < nfault; ++i) {
        const long fc = facets[i];
        FacetInfo const& fi = op->fct[fc];
        const bool boundary = fi.up[0] == fi.up[1];
        // AdapterBase::prepare: oriented normal, its length and the fault mass matrix
        std::vector<double> n(static_cast<size_t>(nq) * D), nl(nq), fq(nq);
        for (int q = 0; q < nq; ++q) {
            double dot = 0.0, n2 = 0.0;
            for (int d = 0; d < D; ++d) {
                const double v = op->Normal[(static_cast<size_t>(fc) * nq + q) * D + d];
                dot += ref_normal[d] * v;
                n2 += v * v;
            }
            nl[q] = std::sqrt(n2);
            for (int d = 0; d < D; ++d)
                n[q * D + d] = (dot < 0 ? -1.0 : 1.0) * op->Normal[(static_cast<size_t>(fc) * nq + q) * D + d];
            double s = 0.0;
            for (int p = 0; p < nbf; ++p) s += e_q[p * nq + q] * slip[i * nbf + p];
            fq[q] = (dot < 0 ? -s : s) * (boundary ? 0.5 : 1.0);  // Adapter::slip sign, bc_boundary halving
        }
        Dense m(nbf, nbf);
        for (int a = 0; a < nbf; ++a)
            for (int b = 0; b < nbf; ++b) {
                double s = 0.0;
                for (int q = 0; q < nq; ++q) s += op->w[q] * nl[q] * e_q[a * nq + q] * e_q[b * nq + q];
                m(a, b) = s;
            }
        Dense mi = tdg::invert(m);
        // grad_u(p, q) = 1/2 (K_Dx_q0 u0 + K_Dx_q1 u1) + c00 (E_q0 u0 - E_q1 u1 - f_q) n_unit, c00 = -penalty
        std::vector<double> tq(nq);
        const double c00 = -op->penalty[fc];
        for (int q = 0; q < nq; ++q) {
            double grad[3] = {0.0, 0.0, 0.0};
            double ev[2] = {0.0, 0.0};
            for (int s = 0; s < (boundary ? 1 : 2); ++s) {
                const double* us = u + static_cast<size_t>(fi.up[s]) * op->bs;
                auto const& Eq = op->E_q[fi.localNo[s]];
                auto const& Dq = op->Dxi_q[fi.localNo[s]];
                const double* KG = &(s == 0 ? op->KG0 : op->KG1)[(static_cast<size_t>(fc) * nq + q) * DD];
                for (int l = 0; l < nbfe; ++l) {
                    ev[s] += Eq[l + static_cast<size_t>(nbfe) * q] * us[l];
                    for (int p = 0; p < D; ++p) {
                        double kd = 0.0;
                        for (int e = 0; e < D; ++e) kd += KG[e + D * p] * Dq[idx3(l, e, q, nbfe, D)];
                        grad[p] += (boundary ? 1.0 : 0.5) * kd * us[l];
                    }
                }
            }
            const double jump = boundary ? (ev[0] - fq[q]) : (ev[0] - ev[1] - fq[q]);
            double gn = 0.0;
            for (int p = 0; p < D; ++p) {
                const double g = grad[p] + c00 * jump * op->UnitNormal[(static_cast<size_t>(fc) * nq + q) * D + p];
                gn += g * n[q * D + p];
            }
            tq[q] = op->w[q] * gn;
        }
        // evaluate_traction: traction(p) = minv(r, p) e_q_T(q, r) w(q) grad_u(k, q) n_q(k, q)
        for (int p = 0; p < nbf; ++p) {
            double t = 0.0;
            for (int r = 0; r < nbf; ++r) {
                double a = 0.0;
                for (int q = 0; q < nq; ++q) a += e_q[r * nq + q] * tq[q];
                t += mi(r, p) * a;
            }
            traction[i * nbf + p] = t;
        }
    }
}

}  // extern "C"

// ---- p-multigrid set-up restated (test side) ------------------------------------------------------
extern "C" {

// NodalInterpolation::assemble (app/localoperator/NodalInterpolation.cpp:8-36): one component's
// block is V_to.leftCols(N2) * VInv_from, V the Dubiner Vandermonde at the warp & blend nodes;
// ModalInterpolation::assemble (app/localoperator/ModalInterpolation.h:31-45): injection of the
// first N2 modal coefficients.  out: [N1][N2].
int orc_mg_interpolation(int D, int kind, int n_to, int n_from, double* out) {
    if (n_to <= n_from || n_from < 0) return -1;
    const int N1 = static_cast<int>(tdg::binom(n_to + D, D)), N2 = static_cast<int>(tdg::binom(n_from + D, D));
    std::fill(out, out + static_cast<size_t>(N1) * N2, 0.0);
    if (kind == kPoisson) {
        for (int l = 0; l < N2; ++l) out[static_cast<size_t>(l) * N2 + l] = 1.0;
        return 0;
    }
    Dense Vto = tdg::vandermonde(D, n_to, tdg::warp_blend_nodes(D, n_to));
    Dense VinvFrom = tdg::invert(tdg::vandermonde(D, n_from, tdg::warp_blend_nodes(D, n_from)));
    for (int k = 0; k < N1; ++k)
        for (int l = 0; l < N2; ++l) {
            double s = 0.0;
            for (int j = 0; j < N2; ++j) s += Vto(k, j) * VinvFrom(j, l);
            out[static_cast<size_t>(k) * N2 + l] = s;
        }
    return 0;
}

// MGConfig::levels (app/common/MGConfig.cpp:11-41); returns the number of levels.
int orc_mg_levels(int strategy, int coarse, int N, int* out) {
    if (N <= coarse) coarse = N > 0 ? N - 1 : 0;
    std::vector<int> lv;
    switch (strategy) {
        case 0: lv = {coarse, N}; break;
        case 1: {
            std::vector<int> down{N};
            while (down.back() > coarse) down.push_back(down.back() / 2);
            if (down.back() != coarse) down.back() = coarse;
            lv.assign(down.rbegin(), down.rend());
            break;
        }
        case 2:
            for (int d = coarse; d <= N; ++d) lv.push_back(d);
            break;
        default: return -1;
    }
    std::copy(lv.begin(), lv.end(), out);
    return static_cast<int>(lv.size());
}

}  // extern "C"

// ---- reference-element tables for building geometry nodes on the test side ------------------------
extern "C" {

// Nodes of degree N (family 0 warp & blend, 1 equidistant) [Nbf][D], and the nodal basis values at
// np points [Nbf][np]: what a test-side mesh builder needs to place Curvilinear's geometry nodes
// without the product library.
int orc_ref_nodes(int D, int N, int family, double* out) {
    Points p = family == 0 ? tdg::warp_blend_nodes(D, N) : tdg::equidistant_nodes(D, N);
    std::memcpy(out, p.data(), p.size() * sizeof(double));
    return 0;
}

int orc_ref_basis(int D, int N, int family, int np, const double* points, double* E) {
    RefSpace sp = RefSpace::nodal(D, N, family == 0 ? tdg::warp_blend_nodes(D, N) : tdg::equidistant_nodes(D, N));
    Points pts(points, points + static_cast<size_t>(np) * D);
    Dense e = sp.eval(pts);
    std::memcpy(E, e.a.data(), e.a.size() * sizeof(double));
    return 0;
}

}  // extern "C"
