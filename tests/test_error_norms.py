"""Error norms of the product (tandem's Error<D>::L2 / H1_semi, src/form/Error.cpp) on the host:

* with the operator's own volume rule they equal the oracle's restatement to 1e-12 (random
  solutions against the manufactured reference, curved and straight, 2D and 3D, both kinds), and
  the rule's points map to the operator's volume coordinates;
* with tandem's error rule (order 20) the errors of oracle solves converge at tandem's bounds
  (L2 order in (N, N+1), H1 semi-norm in (N-1, N); test/conftest.py:61-75);
* projection (Elasticity::project) equals the oracle's weighted inverse mass of the L2 right-hand
  side, and projection / evaluation round-trip discrete functions on affine elements."""
import numpy as np
import pytest

from cases import make_mesh, mms_inputs, product_and_oracle, scenario, tandem_quadrature
from oracle import Oracle
from tandem_b200.operator import DGOperator, ELASTICITY, POISSON
from tandem_b200.refelem import conical_rule


class _Smooth3D:
    """u = sin(pi x) cos(pi y) exp(z / 2) (a 3D reference for the Poisson norms)."""

    @staticmethod
    def solution(X):
        return np.sin(np.pi * X[..., 0]) * np.cos(np.pi * X[..., 1]) * np.exp(0.5 * X[..., 2])

    @staticmethod
    def gradient(X):
        s, c = np.sin(np.pi * X[..., 0]), np.cos(np.pi * X[..., 0])
        sy, cy = np.sin(np.pi * X[..., 1]), np.cos(np.pi * X[..., 1])
        ez = np.exp(0.5 * X[..., 2])
        return np.stack([np.pi * c * cy * ez, -np.pi * s * sy * ez, 0.5 * s * cy * ez], axis=-1)


def _reference(sc, kind, X):
    """Values [E, Q, np] and gradients [E, Q, dim, np] of the manufactured solution at X [E, np, dim]."""
    u, du = sc.solution(X), sc.gradient(X)
    if kind == POISSON:
        return u[:, None, :], np.ascontiguousarray(du.transpose(0, 2, 1)[:, None])
    return np.ascontiguousarray(np.moveaxis(u, -1, 1)), np.ascontiguousarray(du.transpose(0, 2, 3, 1))


@pytest.mark.parametrize("kind,dim,curved", [(POISSON, 2, True), (ELASTICITY, 2, True), (POISSON, 3, False),
                                              (ELASTICITY, 3, True)])
def test_error_norms_match_oracle_on_the_volume_rule(kind, dim, curved):
    n, N = (3, 3) if dim == 2 else (1, 3)
    _, op, orc = product_and_oracle(kind, dim, n, N, curved, True)
    q = tandem_quadrature(dim, N)
    X = op.volume_coords()
    np.testing.assert_allclose(op.rule_coords(q.vol_x), X, atol=1e-14)
    sc = _Smooth3D if (kind == POISSON and dim == 3) else scenario(kind, dim, True)
    ref, refgrad = _reference(sc, kind, X)
    x = np.random.default_rng(dim + 3 * kind).standard_normal(op.ndof) * 0.1
    if kind == POISSON:
        o0, o1 = orc.error_L2(x, sc.solution(X)[..., None]), orc.error_H1_semi(x, sc.gradient(X)[..., None, :])
    else:
        o0, o1 = orc.error_L2(x, sc.solution(X)), orc.error_H1_semi(x, sc.gradient(X))
    e0 = op.error_l2(x, q.vol_x, q.vol_w, ref)
    e1 = op.error_h1_semi(x, q.vol_x, q.vol_w, refgrad)
    assert abs(e0 - o0) <= 1e-12 * o0 and abs(e1 - o1) <= 1e-12 * o1, (e0, o0, e1, o1)


@pytest.mark.parametrize("kind,N", [(POISSON, 3), (ELASTICITY, 2)])
def test_mms_rates_with_tandems_error_rule(kind, N):
    dim = 2
    pts, wts = conical_rule(dim, 20)
    errs = []
    for n in (4, 8):
        m = make_mesh(dim, n, N, True)
        q = tandem_quadrature(dim, N)
        orc = Oracle(m, N, kind, q)
        sc, c0, c1, f, g = mms_inputs(orc, kind, dim, True)
        orc.set_material(c0, c1)
        x, st = orc.cg(orc.rhs(f, g), rtol=1e-12)
        assert st["converged"], st
        op = DGOperator(m, N, kind, q)
        ref, refgrad = _reference(sc, kind, op.rule_coords(pts))
        errs.append((op.error_l2(x, pts, wts, ref), op.error_h1_semi(x, pts, wts, refgrad)))
    r0 = np.log2(errs[0][0] / errs[1][0])
    r1 = np.log2(errs[0][1] / errs[1][1])
    assert N - 0.2 < r0 < N + 1.2, (r0, errs)
    assert N - 1.2 < r1 < N + 0.2, (r1, errs)


@pytest.mark.parametrize("dim,curved", [(2, True), (3, True), (2, False)])
def test_projection_is_the_weighted_inverse_mass_of_the_l2_rhs(dim, curved):
    """project(U_Q) = -apply_inverse_mass(rhs(U_Q)) of the oracle at density 1 (the oracle's
    inverse mass carries the wave operator's -1/rho W/|J|)."""
    n = 3 if dim == 2 else 1
    _, op, orc = product_and_oracle(ELASTICITY, dim, n, 3, curved, True)
    U = np.random.default_rng(dim).standard_normal((op.E, dim, op.Nq))
    ref = -orc.apply_inverse_mass(orc.rhs(U, None))
    np.testing.assert_allclose(op.project(U), ref, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("kind,dim", [(POISSON, 2), (ELASTICITY, 2), (POISSON, 3), (ELASTICITY, 3)])
def test_project_evaluate_round_trip_on_affine_elements(kind, dim):
    """On straight elements the projection of a discrete function's values at the volume points
    returns its coefficients, and evaluate() at the volume points gives those values."""
    n = 3 if dim == 2 else 2
    m = make_mesh(dim, n, 3, False)
    q = tandem_quadrature(dim, 3)
    op = DGOperator(m, 3, kind, q)
    x = np.random.default_rng(kind + dim).standard_normal(op.ndof)
    U = op.evaluate(x, q.vol_x)
    np.testing.assert_allclose(op.project(U), x, atol=1e-11)
    # independent check of evaluate(): the oracle's own error of x against those values vanishes
    orc = Oracle(m, 3, kind, q)
    assert orc.error_L2(x, np.ascontiguousarray(U.transpose(0, 2, 1))) <= 1e-12 * np.linalg.norm(x)
