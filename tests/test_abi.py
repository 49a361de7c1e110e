"""The C ABI: the native library loads, exports every entry point include/tandem_b200.h
declares, and reports invalid calls with error codes and messages (no device work)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from cases import make_mesh, tandem_quadrature
from tandem_b200 import _ffi
from tandem_b200.operator import DGOperator, POISSON

HEADER = Path(__file__).resolve().parents[1] / "include" / "tandem_b200.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]*?\b(tdg_\w+)\s*\(", text, flags=re.M)))


def test_every_declared_symbol_is_exported():
    names = declared()
    assert len(names) >= 20
    L = _ffi.lib()
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(_ffi.SYMBOLS), set(names) - set(_ffi.SYMBOLS)


def test_create_rejects_bad_degree():
    m = make_mesh(2, 2, 4)
    with pytest.raises(_ffi.TdgError, match="TDG_E_INVALID"):
        DGOperator(m, 9, POISSON, tandem_quadrature(2, 4))


def test_create_rejects_bad_topology():
    m = make_mesh(2, 2, 4)
    m.facet_up = m.facet_up.copy()
    m.facet_up[0, 0] = 10_000
    with pytest.raises(_ffi.TdgError, match="bad element"):
        DGOperator(m, 4, POISSON, tandem_quadrature(2, 4))


def test_null_arguments():
    L = _ffi.lib()
    assert L.tdg_create(None, None, 0, None) == -1
    assert b"null" in L.tdg_last_error()
    assert L.tdg_apply(None, 0, None, None, 1, 1, None) == -1
    assert L.tdg_flops_apply(None) == -1


def test_apply_before_material_is_a_state_error():
    op = DGOperator(make_mesh(2, 2, 4), 4, POISSON, tandem_quadrature(2, 4))
    L = _ffi.lib()
    dummy = C.c_void_p(0x1000)
    other = C.c_void_p(0x2000)
    rc = L.tdg_apply(op._h, _ffi.TDG_FP64, dummy, other, 1, op.ndof, None)
    assert rc == -5 and b"set_material" in L.tdg_last_error()
    rc = L.tdg_apply(op._h, _ffi.TDG_FP64, dummy, dummy, 1, op.ndof, None)
    assert rc == -1  # aliasing
    rc = L.tdg_apply(op._h, _ffi.TDG_FP64, dummy, other, 1, op.ndof - 1, None)
    assert rc == -1  # ld too small


def test_counters():
    op = DGOperator(make_mesh(2, 64, 4), 4, POISSON, tandem_quadrature(2, 4))
    op.set_material(np.ones((op.E, op.Nq)))
    # 64 x 64 x 2 triangles, degree 4: 122,880 DOF, 47.2 MFLOP, 14.0 MB per apply
    assert op.ndof == 122_880
    assert abs(op.flops_apply() / 1e6 - 47.2) < 0.1
    assert abs(op.bytes_apply() / 1e6 - 14.0) < 0.1
