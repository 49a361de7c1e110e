"""tdg_gf_traction_update (the Green's-function traction update, SeasQDDiscreteGreenOperator::
update_traction: MatMult(G, S) then VecAXPY with the boundary traction) against the same product
on the host in FP64: 1e-13 relative in the max-norm (summation order differs)."""
import ctypes as C

import numpy as np
import pytest
import torch

from tandem_b200 import _ffi

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.mark.parametrize("n,m,ldg,k,with_tb", [(1280, 1280, 1280, 1, True), (333, 517, 520, 3, True),
                                               (64, 31, 31, 6, False), (1, 1, 1, 1, True), (1000, 130, 131, 9, True)])
def test_traction_update_matches_host_product(n, m, ldg, k, with_tb):
    rng = np.random.default_rng(n + m + k)
    G = rng.standard_normal((n, ldg))
    lds, ldo = m + 5, n + 3
    S = rng.standard_normal((k, lds))
    tb = rng.standard_normal(n)
    t = 0.37
    out = torch.full((k, ldo), float("nan"), dtype=torch.float64, device=DEV)
    Gd, Sd, tbd = (torch.as_tensor(a, device=DEV) for a in (G, S, tb))
    _ffi.check(_ffi.lib().tdg_gf_traction_update(n, m, C.c_void_p(Gd.data_ptr()), ldg, C.c_void_p(Sd.data_ptr()), lds,
                                                 k, C.c_void_p(tbd.data_ptr()) if with_tb else None, t,
                                                 C.c_void_p(out.data_ptr()), ldo,
                                                 C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    ref = S[:, :m] @ G[:, :m].T + (t * tb[None, :] if with_tb else 0.0)
    got = out.cpu().numpy()
    assert np.abs(got[:, :n] - ref).max() <= 1e-13 * np.abs(ref).max()
    assert np.all(np.isnan(got[:, n:]))  # nothing written past n in each state


def test_traction_update_rejects_overlap_and_bad_sizes():
    G = torch.zeros(8, 8, dtype=torch.float64, device=DEV)
    S = torch.zeros(2, 8, dtype=torch.float64, device=DEV)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    L = _ffi.lib()
    assert L.tdg_gf_traction_update(8, 8, p(G), 8, p(S), 8, 2, None, 0.0, p(S), 8, None) == _ffi.ERRORS_BY_NAME["TDG_E_INVALID"]
    assert L.tdg_gf_traction_update(8, 8, p(G), 4, p(S), 8, 1, None, 0.0, p(G), 8, None) == _ffi.ERRORS_BY_NAME["TDG_E_INVALID"]
