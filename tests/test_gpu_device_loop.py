"""Device-looped Krylov blocks and coarse solves (CUDA graph conditional while nodes).

* A captured CG block ends on the device at the iteration where a segment asks for a reliable
  update, so a multigrid solve with graphs takes exactly the iterations of the host-driven solve
  that checks after every iteration, and reaches the same solution; a block-Jacobi solve takes at
  most the iterations of the host-driven one (which checks every 8 iterations).
* The multigrid coarse CG runs as a device loop in blocks of 8 iterations: one V-cycle on the
  default stream equals the V-cycle on a side stream, and the coarse iteration counter grows by a
  multiple of 8.
* Every solve is checked against the oracle's operator."""
import numpy as np
import pytest
import torch

from cases import mms_inputs, product_and_oracle
from tandem_b200.operator import ELASTICITY, FP32, FP64, MIXED, POISSON

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def dev(x):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=DEV)


def rel_res(orc, b, x):
    return np.linalg.norm(b - orc.apply(x.cpu().numpy())) / np.linalg.norm(b)


@pytest.mark.parametrize("kind,dim,n,precision", [(POISSON, 2, 8, FP64), (ELASTICITY, 2, 6, MIXED),
                                                  (ELASTICITY, 3, 2, FP64)])
def test_mg_graph_blocks_match_host_checked_solve(kind, dim, n, precision):
    _, op, orc = product_and_oracle(kind, dim, n, 4, True, True)
    _, _, _, f, g = mms_inputs(op, kind, dim, True)
    b = op.rhs(f, g)
    op.mg_setup(smooth_precision=precision)
    op.set_preconditioner("mg")
    if precision == MIXED:
        op.bjacobi_setup(FP32)
    stream = torch.cuda.Stream()
    out = {}
    for graphs in (False, True):
        x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
        st = op.solve(dev(b), x, precision=precision, rtol=1e-10, max_iterations=400, use_graphs=graphs,
                      stream=stream)
        torch.cuda.synchronize()
        assert st["converged"], (graphs, st)
        assert rel_res(orc, b, x) <= 1.5e-10
        out[graphs] = (st, x.cpu().numpy())
    (s0, x0), (s1, x1) = out[False], out[True]
    assert s1["iterations"] == s0["iterations"], (s0, s1)
    assert s1["outer"] == s0["outer"], (s0, s1)
    assert np.linalg.norm(x1 - x0) <= 1e-12 * np.linalg.norm(x0)


@pytest.mark.parametrize("precision", [FP64, MIXED, FP32])
def test_bjacobi_graph_blocks_stop_on_the_device(precision):
    _, op, orc = product_and_oracle(ELASTICITY, 2, 5, 3, True, True)
    _, _, _, f, g = mms_inputs(op, ELASTICITY, 2, True)
    b = op.rhs(f, g)
    op.bjacobi_setup(FP32 if precision == FP32 else FP64)
    stream = torch.cuda.Stream()
    its = {}
    for graphs in (False, True):
        x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
        st = op.solve(dev(b), x, precision=precision, rtol=1e-10, max_iterations=20000, use_graphs=graphs,
                      stream=stream)
        torch.cuda.synchronize()
        assert st["converged"], (graphs, st)
        assert rel_res(orc, b, x) <= 1.5e-10
        its[graphs] = st["iterations"]
    # the host-driven solve runs whole blocks of 8 past each update point; the device loop stops at
    # the point itself (the trajectories then differ by rounding only)
    assert its[True] <= its[False] + 4, its


def test_coarse_solve_device_loop():
    _, op, _ = product_and_oracle(ELASTICITY, 2, 4, 4, True, True)
    op.mg_setup()
    r = dev(np.random.default_rng(3).standard_normal(op.ndof))
    z0 = torch.zeros_like(r)
    z1 = torch.zeros_like(r)
    c0 = op.mg_info()["coarse_iterations"]
    op.mg_apply(r, z0)  # legacy default stream
    torch.cuda.synchronize()
    c1 = op.mg_info()["coarse_iterations"]
    stream = torch.cuda.Stream()
    op.mg_apply(r, z1, stream=stream)
    stream.synchronize()
    c2 = op.mg_info()["coarse_iterations"]
    assert c1 > c0 and (c1 - c0) % 8 == 0, (c0, c1)
    assert c2 - c1 == c1 - c0, (c0, c1, c2)
    assert torch.equal(z0, z1)
    assert torch.isfinite(z0).all() and z0.abs().max() > 0


@pytest.mark.parametrize("limit", [50, 77])
def test_device_loop_stops_at_the_iteration_limit(limit):
    """A device-looped block never runs past max_iterations: the graph block's limit is the
    remaining count, so a solve that cannot converge in time stops at exactly the limit."""
    _, op, _ = product_and_oracle(ELASTICITY, 2, 5, 3, True, True)
    _, _, _, f, g = mms_inputs(op, ELASTICITY, 2, True)
    b = op.rhs(f, g)
    op.bjacobi_setup(FP64)
    x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    st = op.solve(dev(b), x, precision=FP64, rtol=1e-14, max_iterations=limit, use_graphs=True,
                  stream=torch.cuda.Stream(), check=False)
    torch.cuda.synchronize()
    assert st["iterations"] == limit and not st["converged"], st
    assert np.isfinite(st["rel_residual"]) and st["rel_residual"] < 1.0, st
