"""Fault coupling and discrete Green's functions (Poisson, 2D antiplane) against the oracle's
restatement of tandem's Adapter<Poisson> and Poisson::traction_* (app/localoperator/
PoissonAdapter.cpp, Poisson.cpp:678-723) and against per-column FP64 solves
(SeasQDDiscreteGreenOperator::partial_assemble_discrete_greens_function)."""
import numpy as np
import pytest
import torch

from cases import tandem_quadrature
from oracle import Oracle
from tandem_b200 import mesh as M
from tandem_b200.operator import DGOperator, FP32, FP64, POISSON, Fault, greens_function

pytestmark = pytest.mark.gpu
REF_NORMAL = np.array([1.0, 0.0])


def fault_case(nf=8, length=4.0, width=8.0, depth=6.0, ratio=1.6, degree=4):
    m = M.graded_fault_mesh(num_fault_facets=nf, fault_length=length, width=width, depth=depth, ratio=ratio)
    M.topology(m, m.info["boundary_bc"], m.info["interior_bc"])
    M.geometry_nodes(m, degree)
    q = tandem_quadrature(2, degree)
    op = DGOperator(m, degree, POISSON, q)
    orc = Oracle(m, degree, POISSON, q)
    K = np.ones((op.E, op.Nq))
    op.set_material(K)
    orc.set_material(K)
    facets = M.fault_facets(m)
    return m, op, orc, facets


def test_slip_rhs_matches_oracle():
    m, op, orc, facets = fault_case()
    fl = Fault(op, facets, REF_NORMAL)
    nrhs = 3
    slip = np.random.default_rng(2).standard_normal((nrhs, fl.ncoef))
    b = torch.zeros(nrhs, op.ndof, dtype=torch.float64, device="cuda")
    fl.slip_rhs(torch.as_tensor(slip, device="cuda"), b, nrhs)
    torch.cuda.synchronize()
    for r in range(nrhs):
        ref = orc.rhs(None, orc.fault_slip_q(facets, REF_NORMAL, slip[r].reshape(fl.nfault, fl.nbf)))
        got = b[r].cpu().numpy()
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_traction_matches_oracle():
    m, op, orc, facets = fault_case()
    fl = Fault(op, facets, REF_NORMAL)
    nrhs = 2
    rng = np.random.default_rng(4)
    u = rng.standard_normal((nrhs, op.ndof))
    slip = rng.standard_normal((nrhs, fl.ncoef))
    T = torch.zeros(nrhs, fl.ncoef, dtype=torch.float64, device="cuda")
    fl.traction(torch.as_tensor(u, device="cuda"), torch.as_tensor(slip, device="cuda"), T, nrhs)
    torch.cuda.synchronize()
    for r in range(nrhs):
        ref = orc.fault_traction(facets, REF_NORMAL, u[r], slip[r].reshape(fl.nfault, fl.nbf)).ravel()
        assert np.abs(T[r].cpu().numpy() - ref).max() <= 1e-11 * np.abs(ref).max()


def test_greens_function_batched_matches_per_column_solves():
    m, op, orc, facets = fault_case()
    fl = Fault(op, facets, REF_NORMAL)
    op.bjacobi_setup(FP64)
    G, stats = greens_function(op, fl, FP64, rtol=1e-11)
    assert all(s["converged"] for s in stats)
    Gh = G.cpu().numpy()
    for col in (0, 7, fl.ncoef // 2, fl.ncoef - 1):
        slip = np.zeros(fl.ncoef)
        slip[col] = 1.0
        sl = slip.reshape(fl.nfault, fl.nbf)
        b = orc.rhs(None, orc.fault_slip_q(facets, REF_NORMAL, sl))
        x, st = orc.cg(b, rtol=1e-12)
        assert st["converged"]
        ref = orc.fault_traction(facets, REF_NORMAL, x, sl).ravel()
        assert np.abs(Gh[:, col] - ref).max() <= 1e-8 * np.abs(ref).max(), col


def test_greens_function_mixed_precision():
    m, op, orc, facets = fault_case(nf=16, length=4.0, width=10.0, depth=8.0, ratio=1.3)
    fl = Fault(op, facets, REF_NORMAL)
    op.bjacobi_setup(FP64)
    G64, _ = greens_function(op, fl, FP64, rtol=1e-10)
    op.bjacobi_setup(FP32)
    G32, stats = greens_function(op, fl, FP32, rtol=1e-10, batch=40)
    assert all(s["converged"] for s in stats)
    err = (torch.norm(G32 - G64) / torch.norm(G64)).item()
    assert err < 1e-8, err


def test_greens_operator_resume_and_traction_update(tmp_path):
    """G computed in two sessions through a checkpoint (the second one with the fault facets in
    reverse order) equals G computed in one; update_traction(s, t) = G s + t t_boundary equals the
    traction of the solve with slip s and the boundary data scaled by t."""
    from tandem_b200.greens import DiscreteGreensOperator
    m, op, orc, facets = fault_case(nf=4)
    op.bjacobi_setup(FP64)
    fl = Fault(op, facets, REF_NORMAL)
    full = DiscreteGreensOperator(op, fl)
    full.compute(rtol=1e-12, batch=8)
    ck = str(tmp_path / "gf.npz")
    part = DiscreteGreensOperator(op, fl)
    part.compute(rtol=1e-12, batch=8, checkpoint=ck, max_batches=1)
    assert 0 < part.current < part.n
    rev = Fault(op, facets[::-1].copy(), REF_NORMAL)
    resumed = DiscreteGreensOperator(op, rev)
    assert resumed.load(ck) == part.current
    resumed.compute(rtol=1e-12, batch=8)
    nbf = fl.nbf
    perm = np.arange(fl.nfault)[::-1]
    idx = torch.as_tensor((perm[:, None] * nbf + np.arange(nbf)[None, :]).ravel(), device="cuda")
    Gr = resumed.G[idx][:, idx]
    assert torch.max(torch.abs(Gr - full.G)).item() <= 1e-10 * torch.max(torch.abs(full.G)).item()

    # traction update vs a direct solve
    Xf = op.facet_coords()
    g = np.ascontiguousarray((0.1 * np.cos(Xf[..., 0]) + 0.05 * Xf[..., 1])[:, None, :])
    full.compute_boundary_traction(None, g, rtol=1e-12)
    s = torch.as_tensor(np.random.default_rng(5).standard_normal(fl.ncoef), device="cuda")
    t = 0.7
    b = torch.as_tensor(t * op.rhs(None, g), device="cuda")
    fl.slip_rhs(s, b)
    x = torch.zeros_like(b)
    op.solve(b, x, rtol=1e-12)
    direct = torch.empty(fl.ncoef, dtype=torch.float64, device="cuda")
    fl.traction(x, s, direct)
    upd = full.update_traction(s, t)
    assert torch.max(torch.abs(upd - direct)).item() <= 1e-8 * torch.max(torch.abs(direct)).item()
