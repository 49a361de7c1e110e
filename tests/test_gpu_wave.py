"""Explicit wave operator of elasticity (tandem's Elasticity::wave_rhs and apply_inverse_mass)
against the oracle: the inverse mass to 1e-12, wave_rhs = inverse mass of (A x - b) to 1e-12,
multi-RHS and in place; and the static solution of A u = b has zero acceleration."""
import numpy as np
import pytest
import torch

from cases import make_mesh, material, tandem_quadrature
from oracle import Oracle
from tandem_b200.operator import DGOperator, ELASTICITY

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _case(dim, n, N):
    m = make_mesh(dim, n, N, curved=True)
    q = tandem_quadrature(dim, N)
    op = DGOperator(m, N, ELASTICITY, q)
    orc = Oracle(m, N, ELASTICITY, q)
    c0, c1 = material(ELASTICITY, dim, op.volume_coords(), True)
    op.set_material(c0, c1)
    orc.set_material(c0, c1)
    X = op.volume_coords()
    rho = 1.0 + 0.3 * np.sin(2.0 * X[..., 0] + X[..., 1])
    op.set_density(rho)
    orc.set_density(rho)
    Xf = op.facet_coords()
    g = np.ascontiguousarray(np.stack([0.1 * np.cos(Xf[..., 0] + i) for i in range(dim)], axis=1))
    return m, op, orc, g


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("dim,n,N", [(2, 3, 4), (3, 2, 3)])
def test_inverse_mass_and_wave_rhs_match_oracle(dim, n, N):
    m, op, orc, g = _case(dim, n, N)
    x = np.random.default_rng(dim).standard_normal(op.ndof)
    xd = torch.as_tensor(x, device=DEV)
    y = torch.empty_like(xd)
    op.apply_inverse_mass(xd, y)
    torch.cuda.synchronize()
    assert _rel(y.cpu().numpy(), orc.apply_inverse_mass(x)) < 1e-12
    b = orc.rhs(None, g)
    w = torch.empty_like(xd)
    op.wave_rhs(xd, w, torch.as_tensor(b, device=DEV))
    torch.cuda.synchronize()
    ref = orc.apply_inverse_mass(orc.apply(x) - b)
    assert _rel(w.cpu().numpy(), ref) < 1e-12
    # two right-hand sides, and the inverse mass in place
    X2 = torch.stack([xd, 2.0 * xd])
    Y2 = torch.empty_like(X2)
    op.wave_rhs(X2, Y2, nrhs=2)
    torch.cuda.synchronize()
    ref0 = orc.apply_inverse_mass(orc.apply(x))
    assert _rel(Y2[0].cpu().numpy(), ref0) < 1e-12 and _rel(Y2[1].cpu().numpy(), 2.0 * ref0) < 1e-12
    z = xd.clone()
    op.apply_inverse_mass(z, z)
    torch.cuda.synchronize()
    assert _rel(z.cpu().numpy(), orc.apply_inverse_mass(x)) < 1e-12


def test_static_solution_has_zero_acceleration():
    m, op, orc, g = _case(2, 4, 3)
    b = torch.as_tensor(op.rhs(None, g), device=DEV)
    op.bjacobi_setup(0)
    u = torch.zeros_like(b)
    op.solve(b, u, rtol=1e-12)
    a = torch.empty_like(u)
    op.wave_rhs(u, a, b)
    scale = torch.empty_like(u)
    op.apply_inverse_mass(b, scale)
    torch.cuda.synchronize()
    assert torch.norm(a).item() <= 1e-8 * torch.norm(scale).item()
