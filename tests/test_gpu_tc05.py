"""The 5th-generation tensor-core building blocks of the FP32 operator (tcgen05.mma kind::tf32,
accumulator in tensor memory, core-matrix shared-memory descriptors) through
tdg_probe_tc05_gemm: D = A B^T against an FP64 product of the same FP32 operands.  Tolerances
(max-norm relative to max |A| |B|^T), both operands staged K-major: 3xTF32 2e-6 (about 2^-21 per product, K <= 64 terms),
one TF32 pass 4e-3 (10-bit mantissas)."""
import ctypes as C

import numpy as np
import pytest
import torch

from tandem_b200 import _ffi

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _gemm(A, B, split3):
    n, k = B.shape
    Ad = torch.as_tensor(A, device=DEV)
    Bd = torch.as_tensor(B, device=DEV)
    Dd = torch.full((128, n), float("nan"), dtype=torch.float32, device=DEV)
    _ffi.check(_ffi.lib().tdg_probe_tc05_gemm(C.c_void_p(Ad.data_ptr()), C.c_void_p(Bd.data_ptr()),
                                              C.c_void_p(Dd.data_ptr()), n, k, split3,
                                              C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return Dd.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("n,k", [(16, 8), (48, 40), (96, 16), (176, 64), (256, 64)])
def test_tc05_gemm_3xtf32(n, k):
    rng = np.random.default_rng(n * 100 + k)
    A = rng.standard_normal((128, k)).astype(np.float32)
    B = rng.standard_normal((n, k)).astype(np.float32)
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    scale = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64).T
    D = _gemm(A, B, 1)
    assert np.all(np.isfinite(D))
    assert np.max(np.abs(D - ref) / scale) < 2e-6
    D1 = _gemm(A, B, 0)
    err1 = np.max(np.abs(D1 - ref) / scale)
    assert err1 < 4e-3


def test_tc05_gemm_rejects_bad_shapes():
    A = torch.zeros(128 * 8, device=DEV)
    for n, k in [(8, 8), (24, 8), (272, 8), (16, 4), (16, 72)]:
        rc = _ffi.lib().tdg_probe_tc05_gemm(C.c_void_p(A.data_ptr()), C.c_void_p(A.data_ptr()),
                                            C.c_void_p(A.data_ptr()), n, k, 1, None)
        assert _ffi.ERRORS.get(rc) == "TDG_E_INVALID"


def test_tc05_bounded_wait_reports_timeout():
    """An mbarrier that nothing arrives on: the kernel's bounded wait (about 2 s) runs out, the
    kernel records its status word, frees its tensor memory and returns; the call reports
    TDG_E_TIMEOUT and the context stays usable (a 3xTF32 product right after is correct)."""
    rng = np.random.default_rng(5)
    A = rng.standard_normal((128, 16)).astype(np.float32)
    B = rng.standard_normal((32, 16)).astype(np.float32)
    with pytest.raises(_ffi.TdgError, match="TDG_E_TIMEOUT"):
        _gemm(A, B, -1)
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    scale = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64).T
    assert np.max(np.abs(_gemm(A, B, 1) - ref) / scale) < 2e-6
