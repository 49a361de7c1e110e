"""tandem_b200: the matrix-free SIPG operator of TEAR-ERC/tandem on NVIDIA B200 (sm_100a).

The compute path is the native library ``_lib/libtandem_b200.so`` (C ABI in
``include/tandem_b200.h``); this package holds the host-side mirror of tandem's DG operator
interface (``operator.DGOperator``), mesh/topology tooling and closed-form scenarios.
"""
from . import _ffi  # noqa: F401

__all__ = ["_ffi"]
