"""Device apply against the oracle on meshes that mix every facet code tandem's facet loop branches
on (Poisson.cpp:591-631, Elasticity.cpp:752-801): boundary Dirichlet, Natural (no flux), Fault and
None (the element as its own neighbour), interior Fault (skeleton flux) and interior Natural (a
crack: no flux), see cases.mixed_bc_codes.

Every kernel family is pinned separately (set_apply_config): the face-centric tensor-core pair
(and its software-pipelined form, FP64; with the volume term on tcgen05, FP32), the element-centric
tensor-core kernel and the SIMT kernel.  Tolerances: FP64 1e-12 relative
(max-norm over the vector; summation order differs), FP32 and mixed (FP32 arithmetic on FP64
vectors) 2e-5 relative in the 2-norm."""
import numpy as np
import pytest
import torch

from cases import product_and_oracle
from tandem_b200.operator import ELASTICITY, FP32, FP64, MIXED, POISSON

pytestmark = pytest.mark.gpu
DEV = "cuda:0"

CASES = [
    # kind, dim, n, degree, curved
    (POISSON, 2, 4, 2, True),
    (POISSON, 2, 4, 4, False),
    (POISSON, 3, 2, 2, False),
    (POISSON, 3, 2, 4, True),
    (ELASTICITY, 2, 4, 2, False),
    (ELASTICITY, 2, 4, 4, True),
    (ELASTICITY, 3, 2, 2, True),
    (ELASTICITY, 3, 2, 4, True),
]
IDS = ["k{}d{}n{}p{}c{}".format(*c) for c in CASES]


def rel_max(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def rel_2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module", params=CASES, ids=IDS)
def case(request):
    kind, dim, n, N, curved = request.param
    _, op, orc = product_and_oracle(kind, dim, n, N, curved, True, mixed_bc=True)
    x = np.random.default_rng(17).standard_normal(op.ndof)
    return op, orc, x, orc.apply(x)


@pytest.mark.parametrize("family", ["face", "face2", "tensor", "simt"])
def test_apply_fp64_mixed_bc(case, family):
    op, orc, x, ref = case
    op.set_apply_config(FP64, family)
    y = torch.full((op.ndof,), float("nan"), dtype=torch.float64, device=DEV)
    op.apply(torch.as_tensor(x, device=DEV), y)
    torch.cuda.synchronize()
    assert rel_max(y.cpu().numpy(), ref) < 1e-12


@pytest.mark.parametrize("family", ["face", "tc05", "tensor", "simt"])
def test_apply_fp32_mixed_bc(case, family):
    op, orc, x, _ = case
    op.set_apply_config(FP32, family)
    ref = orc.apply(x.astype(np.float32).astype(np.float64))
    y = torch.full((op.ndof,), float("nan"), dtype=torch.float32, device=DEV)
    op.apply(torch.as_tensor(x, dtype=torch.float32, device=DEV), y, precision=FP32)
    torch.cuda.synchronize()
    assert rel_2(y.cpu().numpy().astype(np.float64), ref) < 2e-5


@pytest.mark.parametrize("family", ["face", "tc05", "tensor"])
def test_apply_mixed_precision_mixed_bc(case, family):
    op, orc, x, ref = case
    op.set_apply_config(FP32, family)
    y = torch.full((op.ndof,), float("nan"), dtype=torch.float64, device=DEV)
    op.apply(torch.as_tensor(x, device=DEV), y, precision=MIXED)
    torch.cuda.synchronize()
    assert rel_2(y.cpu().numpy(), ref) < 2e-5


def test_block_jacobi_blocks_mixed_bc(case):
    """The diagonal blocks (assemble_volume + assemble_skeleton / assemble_boundary per code,
    Poisson.cpp:225-385, Elasticity.cpp:317-519) against the oracle's."""
    op, orc, _, _ = case
    op.bjacobi_setup(FP64)
    assert rel_max(op.bjacobi_blocks(), orc.assemble_diag()) < 1e-12
