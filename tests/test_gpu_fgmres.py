"""Device FGMRES (tdg_solve with TDG_KSP_FGMRES, tandem's -ksp_type fgmres of
examples/options/mg_cheby.cfg) against the oracle: solutions reach the 1e-10 relative residual
of the oracle's operator (FP64 and mixed, multigrid and block-Jacobi preconditioning, multi-RHS
and segmented batches), and agree with the CG solution of the same system to 1e-8 relative when
both are solved to 1e-11."""
import numpy as np
import pytest
import torch

from cases import make_mesh, material, mms_inputs, product_and_oracle, tandem_quadrature
from oracle import Oracle
from tandem_b200 import _ffi
from tandem_b200 import mesh as M
from tandem_b200.operator import DGOperator, ELASTICITY, FP32, FP64, MIXED, POISSON, solve_segmented

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _oracle_rel(orc, b, x):
    return np.linalg.norm(b - orc.apply(x)) / np.linalg.norm(b)


def _config1():
    """64 x 64 x 2 triangles, Poisson p4, K = 1, sin sin MMS (122,880 DOF)."""
    m = make_mesh(2, 64, 4)
    q = tandem_quadrature(2, 4)
    op, orc = DGOperator(m, 4, POISSON, q), Oracle(m, 4, POISSON, q)
    K = np.ones((op.E, op.Nq))
    op.set_material(K)
    orc.set_material(K)
    _, _, _, f, g = mms_inputs(op, POISSON, 2, False)
    return op, orc, op.rhs(f, g)


def _config2_small(n=8):
    """The 3D elasticity cube at n^3 x 6 curved tets, p4, random-field Lame parameters."""
    m = make_mesh(3, n, 4, True)
    q = tandem_quadrature(3, 4)
    op, orc = DGOperator(m, 4, ELASTICITY, q), Oracle(m, 4, ELASTICITY, q)
    c0, c1 = material(ELASTICITY, 3, op.volume_coords(), True, ell=0.2)
    op.set_material(c0, c1)
    orc.set_material(c0, c1)
    _, _, _, f, g = mms_inputs(op, ELASTICITY, 3, True)
    return op, orc, op.rhs(f, g)


@pytest.mark.parametrize("which", ["config1", "config2_8"])
def test_fgmres_multigrid_matches_oracle_and_cg(which):
    op, orc, b = _config1() if which == "config1" else _config2_small()
    op.mg_setup()
    op.set_preconditioner("mg")
    bd = torch.as_tensor(b, device=DEV)
    x = torch.zeros_like(bd)
    st = op.solve(bd, x, precision=FP64, rtol=1e-10, method="fgmres", restart=30)
    assert st["converged"] and st["rel_residual"] <= 1e-10, st
    assert _oracle_rel(orc, b, x.cpu().numpy()) <= 1.5e-10
    # both methods to 1e-11 (near the attainable accuracy of the FP64 residual): the solutions
    # agree to 1e-8
    xg, xc = torch.zeros_like(bd), torch.zeros_like(bd)
    sg = op.solve(bd, xg, precision=FP64, rtol=1e-11, method="fgmres", check=False)
    sc = op.solve(bd, xc, precision=FP64, rtol=1e-11, method="cg", check=False)
    assert sg["rel_residual"] <= 2e-11 and sc["rel_residual"] <= 2e-11, (sg, sc)
    assert (torch.norm(xg - xc) / torch.norm(xc)).item() <= 1e-8


def test_fgmres_mixed_multigrid_reaches_fp64_residual():
    op, orc, b = _config2_small(6)
    op.mg_setup(smooth_precision=MIXED)
    op.set_preconditioner("mg")
    bd = torch.as_tensor(b, device=DEV)
    x = torch.zeros_like(bd)
    st = op.solve(bd, x, precision=MIXED, rtol=1e-10, method="fgmres", restart=20)
    assert st["converged"], st
    assert _oracle_rel(orc, b, x.cpu().numpy()) <= 1.5e-10


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_fgmres_block_jacobi_multi_rhs(precision):
    """Three right-hand sides at a padded leading dimension, block-Jacobi preconditioning, a short
    restart (several cycles): every column reaches 1e-10 on the oracle's operator.  The mesh has a
    Natural top and an interior fault line (an SPD operator, as tandem's scenarios have)."""
    def top_natural(c):
        return np.where(np.all(np.abs(c[:, :, 1] - 1.0) < 1e-9, axis=1), M.BC_NATURAL, M.BC_DIRICHLET)

    def fault(c):
        return np.where(np.all(np.abs(c[:, :, 0] - 0.5) < 1e-9, axis=1), M.BC_FAULT, M.BC_NONE)

    _, op, orc = product_and_oracle(ELASTICITY, 2, 4, 3, True, True, bc=top_natural, interior_bc=fault)
    op.bjacobi_setup(FP64)
    op.set_preconditioner("bjacobi")
    nrhs, ld = 3, op.ndof + 11
    rng = np.random.default_rng(9)
    B = np.zeros((nrhs, ld))
    B[:, :op.ndof] = rng.standard_normal((nrhs, op.ndof))
    X = torch.zeros(nrhs, ld, dtype=torch.float64, device=DEV)
    st = op.solve(torch.as_tensor(B, device=DEV), X, precision=precision, rtol=1e-10, nrhs=nrhs, ld=ld,
                  method="fgmres", restart=12)
    assert st["converged"] and st["outer"] > 1, st
    Xh = X.cpu().numpy()
    for r in range(nrhs):
        assert _oracle_rel(orc, B[r, :op.ndof], Xh[r, :op.ndof]) <= 1.5e-10
        assert np.all(Xh[r, op.ndof:] == 0)


def test_fgmres_segmented_batch():
    meshes = [make_mesh(2, n, 3, curved=True) for n in (2, 5, 3)]
    um, eoff = M.union(meshes)
    q = tandem_quadrature(2, 3)
    op, orc = DGOperator(um, 3, ELASTICITY, q), Oracle(um, 3, ELASTICITY, q)
    c0, c1 = material(ELASTICITY, 2, op.volume_coords(), True)
    op.set_material(c0, c1)
    orc.set_material(c0, c1)
    _, _, _, f, g = mms_inputs(op, ELASTICITY, 2, True)
    b = op.rhs(f, g)
    op.mg_setup()
    op.set_preconditioner("mg")
    x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    st, rel = solve_segmented(op, torch.as_tensor(b, device=DEV), x, eoff, precision=FP64, rtol=1e-10,
                              method="fgmres")
    assert st["converged"] and np.all(rel <= 1e-10), (st, rel)
    r = b - orc.apply(x.cpu().numpy())
    for i in range(len(meshes)):
        sl = slice(eoff[i] * op.bs, eoff[i + 1] * op.bs)
        assert np.linalg.norm(r[sl]) / np.linalg.norm(b[sl]) <= 1.5e-10


def test_fgmres_rejects_fp32_and_long_restart():
    _, op, _ = product_and_oracle(POISSON, 2, 2, 2, False, False)
    op.bjacobi_setup(FP32)
    b = torch.ones(op.ndof, dtype=torch.float64, device=DEV)
    x = torch.zeros_like(b)
    with pytest.raises(_ffi.TdgError, match="TDG_E_INVALID"):
        op.solve(b, x, precision=FP32, method="fgmres")
    op.bjacobi_setup(FP64)
    with pytest.raises(_ffi.TdgError, match="TDG_E_INVALID"):
        op.solve(b, x, precision=FP64, method="fgmres", restart=65)
