"""tdg_apply_host (operator.apply_host): applies on vectors in host memory, streamed through two
device buffer pairs with the copies overlapping the applies, against the device apply of the same
vectors (the same kernels; the facet kernels' atomic additions may land in another order, so
1e-13 relative in FP64 / mixed and 1e-6 in FP32) and the oracle (FP64 1e-12)."""
import numpy as np
import pytest
import torch

from cases import product_and_oracle
from tandem_b200 import _ffi
from tandem_b200.operator import ELASTICITY, FP32, FP64, MIXED, POISSON

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.mark.parametrize("precision", [FP64, FP32, MIXED])
@pytest.mark.parametrize("count,stride_extra", [(1, 0), (5, 0), (5, 7)])
def test_apply_host_matches_device_apply(precision, count, stride_extra):
    _, op, orc = product_and_oracle(ELASTICITY, 3, 2, 3, True, True)
    n = op.ndof
    stride = n + stride_extra
    dt = torch.float32 if precision == FP32 else torch.float64
    rng = np.random.default_rng(count * 10 + stride_extra)
    X = torch.zeros(count * stride, dtype=dt).pin_memory()
    for i in range(count):
        X[i * stride:i * stride + n] = torch.as_tensor(rng.standard_normal(n), dtype=dt)
    Y = torch.full((count * stride,), 7.0, dtype=dt).pin_memory()
    op.apply_host(X, Y, precision=precision, count=count, stride=stride)
    torch.cuda.synchronize()
    for i in range(count):
        xd = X[i * stride:i * stride + n].to(DEV)
        yd = torch.empty_like(xd)
        op.apply(xd, yd, precision=precision)
        torch.cuda.synchronize()
        got, want = Y[i * stride:i * stride + n].double(), yd.cpu().double()
        tol = 1e-6 if precision == FP32 else 1e-13
        assert torch.max(torch.abs(got - want)).item() <= tol * torch.max(torch.abs(want)).item()
        if stride_extra:
            assert torch.all(Y[i * stride + n:(i + 1) * stride] == 7.0)
    if precision == FP64:
        ref = orc.apply(X[:n].numpy())
        assert np.abs(Y[:n].numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


def test_apply_host_same_vector_every_time():
    _, op, orc = product_and_oracle(POISSON, 2, 4, 3, True, True)
    n = op.ndof
    x = torch.as_tensor(np.random.default_rng(3).standard_normal(n)).pin_memory()
    y = torch.zeros(n, dtype=torch.float64).pin_memory()
    op.apply_host(x, y, count=4, stride=0)
    torch.cuda.synchronize()
    ref = orc.apply(x.numpy())
    assert np.abs(y.numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


def test_apply_host_rejects_bad_arguments():
    _, op, _ = product_and_oracle(POISSON, 2, 2, 2, False, False)
    x = torch.zeros(op.ndof, dtype=torch.float64)
    with pytest.raises(_ffi.TdgError, match="TDG_E_INVALID"):
        _ffi.check(_ffi.lib().tdg_apply_host(op._h, FP64, x.data_ptr(), x.data_ptr(), 1, 0, None))
    with pytest.raises(_ffi.TdgError, match="TDG_E_INVALID"):
        _ffi.check(_ffi.lib().tdg_apply_host(op._h, FP64, x.data_ptr(), x.data_ptr() + 8, 1, 3, None))
