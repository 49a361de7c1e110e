"""One-pass TF32 operator (TDG_TF32) and the multigrid smoother that uses it.

* TDG_TF32 applies the operator on FP64 vectors with one TF32 tensor-core pass per product: it
  agrees with the oracle to 1e-2 relative (2-norm; a TF32 operand keeps 10 mantissa bits), is
  less accurate than the 3xTF32 apply of the same kernels (TDG_MIXED, 2e-5) -- so the one-pass
  kernels are the ones that ran -- for the element-centric, face-centric and tcgen05 families.
* A mixed multigrid solve whose finest-level smoother applies run in TDG_TF32 reaches the 1e-10
  FP64 residual of the oracle's operator, in at most 25 % more iterations than with the 3xTF32
  smoother."""
import numpy as np
import pytest
import torch

from cases import mms_inputs, product_and_oracle
from tandem_b200.operator import ELASTICITY, FP32, FP64, MIXED, POISSON, TF32

pytestmark = pytest.mark.gpu
DEV = "cuda:0"

CASES = [
    # kind, dim, n, degree, curved, variable
    (POISSON, 2, 4, 4, False, False),
    (POISSON, 3, 2, 4, True, True),
    (ELASTICITY, 2, 3, 4, True, True),
    (ELASTICITY, 3, 2, 4, True, True),
    (ELASTICITY, 3, 2, 2, True, True),
]


def dev(x):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=DEV)


@pytest.mark.parametrize("family", ["tensor", "face", "tc05"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "k{}d{}n{}p{}c{}v{}".format(*c))
def test_tf32_apply_close_to_oracle(case, family):
    kind, dim, n, N, curved, var = case
    _, op, orc = product_and_oracle(kind, dim, n, N, curved, var)
    op.set_apply_config(FP32, family, 2)
    x = np.random.default_rng(11).standard_normal(op.ndof)
    ref = orc.apply(x.astype(np.float32).astype(np.float64))
    err = {}
    for prec in (MIXED, TF32):
        y = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
        op.apply(dev(x), y, precision=prec)
        torch.cuda.synchronize()
        err[prec] = np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err[MIXED] < 2e-5, err
    assert err[TF32] < 1e-2, err
    assert err[TF32] > err[MIXED], err


@pytest.mark.parametrize("kind,dim,n", [(POISSON, 2, 8), (ELASTICITY, 2, 6), (ELASTICITY, 3, 2)])
def test_mg_solve_with_tf32_smoother(kind, dim, n):
    _, op, orc = product_and_oracle(kind, dim, n, 4, True, True)
    _, _, _, f, g = mms_inputs(op, kind, dim, True)
    b = op.rhs(f, g)
    op.set_preconditioner("mg")
    its = {}
    for smooth in (MIXED, TF32):
        op.mg_setup(smooth_precision=smooth)
        x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
        st = op.solve(dev(b), x, precision=MIXED, rtol=1e-10, max_iterations=400)
        torch.cuda.synchronize()
        assert st["converged"] and st["rel_residual"] <= 1e-10, (smooth, st)
        assert np.linalg.norm(b - orc.apply(x.cpu().numpy())) / np.linalg.norm(b) <= 1.5e-10
        its[smooth] = st["iterations"]
    assert its[TF32] <= 1.25 * its[MIXED] + 2, its


def test_tf32_is_not_a_solve_precision():
    from tandem_b200 import _ffi
    _, op, _ = product_and_oracle(POISSON, 2, 3, 2, False, False)
    b = torch.ones(op.ndof, dtype=torch.float64, device=DEV)
    x = torch.zeros_like(b)
    op.bjacobi_setup(FP64)
    with pytest.raises(_ffi.TdgError, match="TDG_E_INVALID"):
        op.solve(b, x, precision=TF32)
