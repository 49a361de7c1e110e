"""tdg_update_material: the material changes, the preconditioner built for the previous one stays.

The apply after an update equals the apply after tdg_set_material with the same material
(bit-identical: the same host set-up and upload), and a solve preconditioned by the kept
block-Jacobi inverses or multigrid hierarchy reaches the 1e-10 FP64 residual of the new operator,
checked through the oracle."""
import numpy as np
import pytest
import torch

from cases import make_mesh, material, mms_inputs, tandem_quadrature
from oracle import Oracle
from tandem_b200 import _ffi
from tandem_b200.operator import DGOperator, ELASTICITY, FP64, MIXED

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _op(dim, n, N):
    m = make_mesh(dim, n, N, True)
    q = tandem_quadrature(dim, N)
    op = DGOperator(m, N, ELASTICITY, q)
    c0, c1 = material(ELASTICITY, dim, op.volume_coords(), True)
    op.set_material(c0, c1)
    return m, q, op, c0, c1


def test_update_needs_a_preconditioner():
    _, _, op, c0, c1 = _op(2, 2, 2)
    with pytest.raises(_ffi.TdgError, match="TDG_E_STATE"):
        op.update_material(c0, c1)


@pytest.mark.parametrize("pc,precision", [("bjacobi", FP64), ("mg", FP64), ("mg", MIXED)])
def test_solve_with_kept_preconditioner(pc, precision):
    dim, n, N = 3, 2, 4
    m, q, op, c0, c1 = _op(dim, n, N)
    if pc == "mg":
        op.mg_setup()
        op.set_preconditioner("mg")
    else:
        op.bjacobi_setup(FP64)
    # a 5 % perturbation of every element's material
    rng = np.random.default_rng(4)
    s0 = 1.0 + 0.05 * rng.uniform(-1, 1, (op.E, 1))
    s1 = 1.0 + 0.05 * rng.uniform(-1, 1, (op.E, 1))
    op.update_material(c0 * s0, c1 * s1)
    ref_op = DGOperator(m, N, ELASTICITY, q)
    ref_op.set_material(c0 * s0, c1 * s1)
    x = torch.randn(op.ndof, dtype=torch.float64, device=DEV, generator=torch.Generator(device=DEV).manual_seed(2))
    y, yr = torch.empty_like(x), torch.empty_like(x)
    op.apply(x, y)
    ref_op.apply(x, yr)
    torch.cuda.synchronize()
    assert torch.equal(y, yr)
    orc = Oracle(m, N, ELASTICITY, q)
    orc.set_material(c0 * s0, c1 * s1)
    _, _, _, f, g = mms_inputs(op, ELASTICITY, dim, True)
    b = orc.rhs(f, g)
    xs = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    st = op.solve(torch.as_tensor(b, device=DEV), xs, precision=precision, rtol=1e-10)
    assert st["converged"], st
    r = b - orc.apply(xs.cpu().numpy())
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.5e-10
