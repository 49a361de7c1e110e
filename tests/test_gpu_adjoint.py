"""Adjoint gradient of a displacement misfit with respect to per-element Lame parameters against
central finite differences of the oracle (dense direct solves of the oracle's operator and
right-hand side at perturbed parameters).

Tolerance: |<grad, delta> - FD| <= 1e-6 |FD| + 2e-9 J for every direction.  FD step h = 1e-4:
the truncation error is O(h^2) ~ 1e-8 relative; the dense solves reproduce J to ~1e-13 J, which
puts a noise floor of ~1e-9 J on the central difference (the absolute term; it matters only for
the single-element directions, whose derivatives are small)."""
import numpy as np
import pytest
import torch

from cases import tandem_quadrature
from oracle import Oracle
from tandem_b200 import mesh as M
from tandem_b200.adjoint import LameProblem, lame_solve
from tandem_b200.operator import DGOperator, ELASTICITY

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _mesh(dim, n, degree):
    """Top natural, left boundary a fault (dim 2), other boundaries Dirichlet; an interior fault on
    x = 1/2 (dim 2)."""
    def boundary_bc(c):
        top = np.all(np.abs(c[:, :, dim - 1] - 1.0) < 1e-9, axis=1)
        left = np.all(np.abs(c[:, :, 0]) < 1e-9, axis=1)
        codes = np.where(top, M.BC_NATURAL, M.BC_DIRICHLET)
        return np.where(left & (dim == 2), M.BC_FAULT, codes)

    def interior_bc(c):
        on = np.all(np.abs(c[:, :, 0] - 0.5) < 1e-9, axis=1)
        return np.where(on & (dim == 2), M.BC_FAULT, M.BC_NONE)

    m = M.square_mesh(n) if dim == 2 else M.cube_mesh(n)
    return M.build(m, degree, boundary_bc=boundary_bc, interior_bc=interior_bc,
                   curve=M.box_boundary_surface(0.02))


def _data(op):
    X, Xf = op.volume_coords(), op.facet_coords()
    D = op.dim
    f = np.stack([np.sin(np.pi * X[..., 0] + i) * np.cos(2 * X[..., 1]) for i in range(D)], axis=1)
    g = np.stack([0.1 * np.cos(3 * Xf[..., 0] - i) + 0.05 * Xf[..., 1] for i in range(D)], axis=1)
    return np.ascontiguousarray(f), np.ascontiguousarray(g)


def _theta(op):
    c = op.volume_coords().mean(axis=1)
    lam = 2.0 + 0.5 * np.sin(3 * c[:, 0] + c[:, 1])
    mu = 1.0 + 0.3 * np.cos(2 * c[:, 1] - c[:, 0])
    return lam, mu


class OracleMisfit:
    """J(lam, mu) = 1/2 |u - d|^2 with u from a dense direct solve of the oracle's system."""

    def __init__(self, m, degree, q, f, g, d):
        self.orc = Oracle(m, degree, ELASTICITY, q)
        self.f, self.g, self.d = f, g, d

    def __call__(self, lam, mu):
        o = self.orc
        Nq = self.f.shape[2]
        o.set_material(np.repeat(lam[:, None], Nq, 1), np.repeat(mu[:, None], Nq, 1))
        n = o.ndof
        A = np.empty((n, n))
        e = np.zeros(n)
        for j in range(n):
            e[j] = 1.0
            A[:, j] = o.apply(e)
            e[j] = 0.0
        u = np.linalg.solve(A, o.rhs(self.f, self.g))
        return 0.5 * np.sum((u - self.d) ** 2)


@pytest.mark.parametrize("dim,n,degree", [(2, 4, 2), (2, 3, 3), (3, 2, 2)])
def test_lame_gradient_matches_finite_differences(dim, n, degree):
    m = _mesh(dim, n, degree)
    q = tandem_quadrature(dim, degree)
    op = DGOperator(m, degree, ELASTICITY, q)
    f, g = _data(op)
    lam0, mu0 = _theta(op)
    pb = LameProblem(op, f, g, rtol=1e-13)
    rng = np.random.default_rng(dim * 10 + degree)
    d = torch.as_tensor(rng.standard_normal(op.ndof) * 0.05, device=DEV)

    lam = torch.tensor(lam0, dtype=torch.float64, requires_grad=True)
    mu = torch.tensor(mu0, dtype=torch.float64, requires_grad=True)
    u = lame_solve(lam, mu, pb)
    J = 0.5 * torch.sum((u - d) ** 2)
    J.backward()
    gl, gm = lam.grad.numpy(), mu.grad.numpy()
    assert np.all(np.isfinite(gl)) and np.all(np.isfinite(gm))

    Jo = OracleMisfit(m, degree, q, f, g, d.cpu().numpy())
    assert abs(Jo(lam0, mu0) - J.item()) <= 1e-8 * J.item()
    dirs = [(rng.standard_normal(op.E), np.zeros(op.E)), (np.zeros(op.E), rng.standard_normal(op.E)),
            (rng.standard_normal(op.E), rng.standard_normal(op.E))]
    e_fault = int(m.facet_up[np.nonzero(m.facet_bc == M.BC_FAULT)[0][0], 0]) if dim == 2 else 0
    unit = np.zeros(op.E)
    unit[e_fault] = 1.0
    dirs += [(unit, np.zeros(op.E)), (np.zeros(op.E), unit)]
    h = 1e-4
    for dl, dm in dirs:
        fd = (Jo(lam0 + h * dl, mu0 + h * dm) - Jo(lam0 - h * dl, mu0 - h * dm)) / (2 * h)
        ad = gl @ dl + gm @ dm
        assert abs(ad - fd) <= 1e-6 * abs(fd) + 2e-9 * J.item(), (ad, fd)


def test_gradient_without_boundary_data_is_operator_part_only():
    """With b independent of theta (no boundary data) the gradient is -p^T dA/dtheta u, which for
    p = u (J = 1/2 u^T A u, dJ/du = A u) reduces to -u^T dA/dtheta u; check against d/dtheta of
    u^T A(theta) u at fixed u by central differences of device applies."""
    dim, degree = 2, 3
    m = _mesh(dim, 3, degree)
    q = tandem_quadrature(dim, degree)
    op = DGOperator(m, degree, ELASTICITY, q)
    lam0, mu0 = _theta(op)
    pb = LameProblem(op, None, None, rtol=1e-12)
    pb.set_parameters(lam0, mu0)
    u = torch.as_tensor(np.random.default_rng(4).standard_normal(op.ndof), device=DEV)
    g = pb.gradient(u, u).cpu().numpy()

    def quad(lam, mu):
        pb.set_parameters(lam, mu)
        y = torch.empty_like(u)
        op.apply(u, y)
        return torch.dot(u, y).item()

    rng = np.random.default_rng(9)
    for _ in range(3):
        dl, dm = rng.standard_normal(op.E), rng.standard_normal(op.E)
        h = 1e-5
        fd = (quad(lam0 + h * dl, mu0 + h * dm) - quad(lam0 - h * dl, mu0 - h * dm)) / (2 * h)
        ad = -(g[:, 0] @ dl + g[:, 1] @ dm)
        assert abs(ad - fd) <= 1e-7 * abs(fd), (ad, fd)


def test_variable_material_is_rejected():
    m = _mesh(2, 2, 2)
    q = tandem_quadrature(2, 2)
    op = DGOperator(m, 2, ELASTICITY, q)
    X = op.volume_coords()
    op.set_material(2.0 + X[..., 0], np.ones(X.shape[:2]))
    pb = LameProblem(op)
    u = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    from tandem_b200 import _ffi
    with pytest.raises(_ffi.TdgError, match="not constant per element"):
        pb.gradient(u, u)


def test_multigrid_preconditioned_gradient_equals_block_jacobi():
    """The same gradient (to the solve tolerance) whichever preconditioner the forward and adjoint
    solves use; the mesh has an interior and a boundary fault."""
    dim, degree = 2, 3
    m = _mesh(dim, 4, degree)
    q = tandem_quadrature(dim, degree)
    op = DGOperator(m, degree, ELASTICITY, q)
    f, g = _data(op)
    lam0, mu0 = _theta(op)
    d = torch.as_tensor(np.random.default_rng(3).standard_normal(op.ndof) * 0.05, device=DEV)
    grads = []
    for pc in ("bjacobi", "mg"):
        pb = LameProblem(op, f, g, rtol=1e-12, preconditioner=pc)
        lam = torch.tensor(lam0, dtype=torch.float64, requires_grad=True)
        mu = torch.tensor(mu0, dtype=torch.float64, requires_grad=True)
        u = lame_solve(lam, mu, pb)
        J = 0.5 * torch.sum((u - d) ** 2)
        J.backward()
        grads.append(np.concatenate([lam.grad.numpy(), mu.grad.numpy()]))
        if pc == "mg":
            assert max(s["iterations"] for s in pb.last_stats) < 200, pb.last_stats
    op.set_preconditioner("bjacobi")
    assert np.abs(grads[0] - grads[1]).max() <= 1e-8 * np.abs(grads[0]).max()
