"""tdg_adjoint_lame_gradient_noalloc (fixed device scratch, no allocation) against the allocating
tdg_adjoint_lame_gradient: two calls in a row agree with it to 1e-13 relative (same kernel and
inputs; only where the penalty derivatives are staged differs), and a first call made before any
allocating gradient call leaves the device's free memory unchanged.  The entry point serves
callers that cannot allocate at the time of the call, e.g. an inversion loop in a process whose
caching allocator already holds the device memory.  Collected last on purpose: it must pass after
every other test has run in the process, and alone."""
import numpy as np
import pytest
import torch

from cases import tandem_quadrature
from tandem_b200 import _ffi
from tandem_b200 import mesh as M
from tandem_b200.adjoint import LameProblem
from tandem_b200.operator import DGOperator, ELASTICITY

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _problem(dim, n, degree, with_bc):
    def boundary_bc(c):
        top = np.all(np.abs(c[:, :, dim - 1] - 1.0) < 1e-9, axis=1)
        return np.where(top, M.BC_NATURAL, M.BC_DIRICHLET)

    def interior_bc(c):
        on = np.all(np.abs(c[:, :, 0] - 0.5) < 1e-9, axis=1)
        return np.where(on, M.BC_FAULT, M.BC_NONE)

    m = M.square_mesh(n) if dim == 2 else M.cube_mesh(n)
    m = M.build(m, degree, boundary_bc=boundary_bc, interior_bc=interior_bc, curve=M.box_boundary_surface(0.02))
    op = DGOperator(m, degree, ELASTICITY, tandem_quadrature(dim, degree))
    c = op.volume_coords().mean(axis=1)
    lam = 2.0 + 0.5 * np.sin(3 * c[:, 0] + c[:, 1])
    mu = 1.0 + 0.3 * np.cos(2 * c[:, 1] - c[:, 0])
    g = None
    if with_bc:
        Xf = op.facet_coords()
        g = np.stack([0.1 * np.cos(3 * Xf[..., 0] - i) for i in range(dim)], axis=1)
    pb = LameProblem(op, None, g)
    pb.set_parameters(lam, mu)
    gen = torch.Generator(device=DEV).manual_seed(dim * 100 + n)
    u = torch.randn(op.ndof, dtype=torch.float64, device=DEV, generator=gen)
    p = torch.randn(op.ndof, dtype=torch.float64, device=DEV, generator=gen)
    y = torch.empty_like(u)
    op.apply(u, y)  # makes the FP64 operator data resident
    torch.cuda.synchronize()
    return op, pb, u, p


@pytest.mark.parametrize("dim,n,degree,with_bc", [(2, 6, 3, True), (3, 3, 2, True), (3, 2, 4, False)])
def test_noalloc_gradient_matches_allocating_entry(dim, n, degree, with_bc):
    op, pb, u, p = _problem(dim, n, degree, with_bc)
    ref = pb.gradient(u, p)
    scale = ref.abs().max().item()
    for _ in range(2):  # two calls in a row reuse the same scratch
        g = torch.full((op.E, 2), float("nan"), dtype=torch.float64, device=DEV)
        pb.gradient_noalloc(u, p, g)
        torch.cuda.synchronize()
        assert (g - ref).abs().max().item() <= 1e-13 * scale


@pytest.mark.parametrize("dim,n,degree", [(3, 2, 4), (2, 5, 2)])
def test_noalloc_gradient_first_call_allocates_nothing(dim, n, degree):
    """A fresh operator: one FP64 apply (which uploads the operator, resolves the scratch and loads
    the gradient kernel), then the allocation-free call before any allocating gradient call.  The
    device's free memory is the same before and after it; the result then matches the allocating
    entry point."""
    op, pb, u, p = _problem(dim, n, degree, True)
    g = torch.full((op.E, 2), float("nan"), dtype=torch.float64, device=DEV)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    pb.gradient_noalloc(u, p, g)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 >= free0, (free0, free1)
    ref = pb.gradient(u, p)
    assert (g - ref).abs().max().item() <= 1e-13 * ref.abs().max().item()


def test_noalloc_gradient_needs_resident_operator_data():
    m = M.build(M.square_mesh(2), 2)
    op = DGOperator(m, 2, ELASTICITY, tandem_quadrature(2, 2))
    op.set_material(2.0 * np.ones((op.E, op.Nq)), np.ones((op.E, op.Nq)))
    pb = LameProblem(op)
    u = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    g = torch.zeros(op.E, 2, dtype=torch.float64, device=DEV)
    with pytest.raises(_ffi.TdgError, match="not resident"):
        pb.gradient_noalloc(u, u, g)


def test_noalloc_gradient_rejects_meshes_beyond_the_scratch():
    """300 x 300 x 2 triangles: 4 F + 2 E = 1,442,400 > 2^20 doubles."""
    m = M.build(M.square_mesh(300), 1)
    op = DGOperator(m, 1, ELASTICITY, tandem_quadrature(2, 1))
    op.set_material(2.0 * np.ones((op.E, op.Nq)), np.ones((op.E, op.Nq)))
    assert 4 * op.F + 2 * op.E > 2 ** 20
    pb = LameProblem(op)
    u = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    g = torch.zeros(op.E, 2, dtype=torch.float64, device=DEV)
    with pytest.raises(_ffi.TdgError, match="fixed scratch holds 1048576"):
        pb.gradient_noalloc(u, u, g)
