"""Pins of the oracle itself: tandem's MMS convergence bounds (test/conftest.py:61-75 with the
slope fit of test/test_convergence_static.py:46-67), symmetry of SIPG (MAT_SYMMETRIC,
app/common/PetscDGMatrix.cpp:76), matrix-free apply == assembled diagonal blocks, A 1 = 0 for the
pure-Neumann Poisson operator, and the host right-hand side of the product against the oracle's."""
import numpy as np
import pytest

from cases import make_mesh, mms_inputs, product_and_oracle, tandem_quadrature
from oracle import Oracle
from tandem_b200 import mesh as M
from tandem_b200.operator import DGOperator, POISSON, ELASTICITY


def _solve_mms(kind, dim, n, degree, curved, variable):
    m = make_mesh(dim, n, degree, curved)
    q = tandem_quadrature(dim, degree)
    orc = Oracle(m, degree, kind, q)
    sc, c0, c1, f, g = mms_inputs(orc, kind, dim, variable)
    orc.set_material(c0, c1)
    b = orc.rhs(f, g)
    x, st = orc.cg(b, rtol=1e-12)
    assert st["converged"], st
    X = orc.volume_coords()
    if kind == POISSON:
        e0 = orc.error_L2(x, sc.solution(X)[..., None])
        e1 = orc.error_H1_semi(x, sc.gradient(X)[..., None, :])
    else:
        e0 = orc.error_L2(x, sc.solution(X))
        e1 = orc.error_H1_semi(x, sc.gradient(X))
    return e0, e1


@pytest.mark.parametrize("kind,dim,curved,variable,ns", [
    (POISSON, 2, False, False, (4, 8)),
    (ELASTICITY, 2, True, True, (4, 8)),
])
def test_mms_convergence_rates(kind, dim, curved, variable, ns):
    N = 4
    errs = [_solve_mms(kind, dim, n, N, curved, variable) for n in ns]
    r0 = np.log2(errs[0][0] / errs[1][0])
    r1 = np.log2(errs[0][1] / errs[1][1])
    # tandem's bounds: L2 order in (N, N+1), H1 order in (N-1, N); small pre-asymptotic slack
    assert N - 0.2 < r0 < N + 1.2, (r0, errs)
    assert N - 1.2 < r1 < N + 0.2, (r1, errs)


@pytest.mark.parametrize("kind,dim,curved", [(POISSON, 2, False), (ELASTICITY, 2, True), (POISSON, 3, True),
                                              (ELASTICITY, 3, False)])
def test_symmetric_and_blocks_consistent(kind, dim, curved):
    n = 2 if dim == 2 else 1
    m, op, orc = product_and_oracle(kind, dim, n, 3, curved, True)
    N = orc.ndof
    A = np.stack([orc.apply(np.eye(N)[i]) for i in range(N)], axis=1)
    assert np.abs(A - A.T).max() <= 1e-12 * np.abs(A).max()
    blocks = orc.assemble_diag()
    bs = orc.bs
    for e in range(orc.E):
        np.testing.assert_allclose(A[e * bs:(e + 1) * bs, e * bs:(e + 1) * bs], blocks[e],
                                   atol=1e-12 * np.abs(A).max())
    assert np.linalg.eigvalsh(0.5 * (A + A.T)).min() > 0


def test_neumann_poisson_annihilates_constants():
    m = make_mesh(2, 3, 4, False, bc=M.BC_NATURAL)
    q = tandem_quadrature(2, 4)
    orc = Oracle(m, 4, POISSON, q)
    orc.set_material(np.ones((orc.E, orc.Nq)))
    x = np.zeros(orc.ndof)
    x[::orc.bs] = 1.0  # modal basis: Dubiner P_0 = 1
    assert np.abs(orc.apply(x)).max() < 1e-12


def test_neumann_elasticity_annihilates_translations():
    m = make_mesh(3, 1, 2, True, bc=M.BC_NATURAL)
    q = tandem_quadrature(3, 2)
    orc = Oracle(m, 2, ELASTICITY, q)
    X = orc.volume_coords()
    orc.set_material(2.0 * np.ones(X.shape[:2]), np.ones(X.shape[:2]))
    for c in range(3):
        x = np.zeros((orc.E, 3, orc.nbf))
        x[:, c, :] = 1.0  # nodal basis: constant displacement in component c
        assert np.abs(orc.apply(x.ravel())).max() < 1e-11


@pytest.mark.parametrize("kind,dim", [(POISSON, 2), (ELASTICITY, 2), (ELASTICITY, 3)])
def test_product_rhs_matches_oracle(kind, dim):
    m, op, orc = product_and_oracle(kind, dim, 3 if dim == 2 else 2, 4, True, True)
    sc, c0, c1, f, g = mms_inputs(op, kind, dim, True)
    b_op = op.rhs(f, g)
    b_or = orc.rhs(f, g)
    np.testing.assert_allclose(b_op, b_or, rtol=0, atol=1e-12 * np.abs(b_or).max())


@pytest.mark.parametrize("kind,dim,degree", [(POISSON, 2, 4), (POISSON, 3, 2), (ELASTICITY, 2, 4),
                                             (ELASTICITY, 3, 3)])
def test_product_rhs_matches_oracle_mixed_bc(kind, dim, degree):
    """Every facet code at once (boundary Dirichlet / Natural / Fault / None, interior Fault and
    Natural): the volume load plus the lift terms of rhs_skeleton / rhs_boundary (Poisson.cpp:387-549,
    Elasticity.cpp:521-696), boundary faults with the halved slip."""
    m, op, orc = product_and_oracle(kind, dim, 4 if dim == 2 else 2, degree, True, True, mixed_bc=True)
    sc, c0, c1, f, g = mms_inputs(op, kind, dim, True)
    b_op = op.rhs(f, g)
    b_or = orc.rhs(f, g)
    np.testing.assert_allclose(b_op, b_or, rtol=0, atol=1e-12 * np.abs(b_or).max())


def test_fault_facets_rhs():
    """A fault line through the square: interior facets with BC::Fault use the skeleton lift on
    both sides (Poisson.cpp:434-482); the product's host RHS matches the oracle."""
    fault = lambda c: np.where(np.all(np.abs(c[:, :, 0] - 0.5) < 1e-12, axis=1), M.BC_FAULT, M.BC_NONE)  # noqa: E731
    m = make_mesh(2, 4, 3, False, interior_bc=fault)
    assert (m.facet_bc == M.BC_FAULT).sum() == 4
    q = tandem_quadrature(2, 3)
    op = DGOperator(m, 3, POISSON, q)
    orc = Oracle(m, 3, POISSON, q)
    op.set_material(np.ones((op.E, op.Nq)))
    orc.set_material(np.ones((op.E, op.Nq)))
    g = np.ones((op.F, 1, op.nq))
    np.testing.assert_allclose(op.rhs(None, g), orc.rhs(None, g), atol=1e-12)


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_inverse_mass_inverts_the_mass_on_affine_elements(dim):
    """The -(1/rho)-weighted inverse mass of Elasticity::wave_rhs is the exact element inverse mass
    on affine elements: applied to the load of a nodal field it returns minus the field / rho."""
    from cases import make_mesh, tandem_quadrature
    from tandem_b200 import refelem
    from tandem_b200.operator import ELASTICITY
    N = 3
    m = make_mesh(dim, 2, N, False)
    q = tandem_quadrature(dim, N)
    o = Oracle(m, N, ELASTICITY, q)
    X = o.volume_coords()
    o.set_material(2.0 + X[..., 0], np.ones(X.shape[:2]))
    o.set_density(np.full(X.shape[:2], 2.0))
    EQ = refelem.ref_basis(dim, N, refelem.WARP_BLEND, q.vol_x)
    u = np.random.default_rng(dim).standard_normal(o.ndof)
    fQ = np.einsum("epk,kq->epq", u.reshape(o.E, dim, -1), EQ)
    y = o.apply_inverse_mass(o.rhs(fQ, None))
    assert np.abs(y + 0.5 * u).max() <= 1e-12 * np.abs(u).max()
