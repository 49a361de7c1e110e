"""Reference-element tables from the native library (host-only entry points)."""
from __future__ import annotations

from math import comb

import numpy as np

from . import _ffi

WARP_BLEND, EQUIDISTANT, MODAL = 0, 1, -1


def _ptr(a: np.ndarray):
    return a.ctypes.data if a is not None else None


def ref_nodes(dim: int, degree: int, family: int = WARP_BLEND) -> np.ndarray:
    out = np.zeros((comb(degree + dim, dim), dim))
    _ffi.check(_ffi.lib().tdg_ref_nodes(dim, degree, family, _ptr(out)))
    return out


def ref_basis(dim: int, degree: int, family: int, points: np.ndarray, grad: bool = False):
    """Basis values E[k, q] (and gradients G[k, d, q]) at points [np, dim]."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, dim)
    nbf = comb(degree + dim, dim)
    E = np.zeros((nbf, pts.shape[0]))
    G = np.zeros((nbf, dim, pts.shape[0])) if grad else None
    _ffi.check(_ffi.lib().tdg_ref_basis(dim, degree, family, pts.shape[0], _ptr(pts), _ptr(E), _ptr(G)))
    return (E, G) if grad else E


def conical_rule(dim: int, order: int):
    n = _ffi.lib().tdg_conical_rule(dim, order, None, None)
    if n < 0:
        _ffi.check(n)
    x = np.zeros((n, dim))
    w = np.zeros(n)
    _ffi.lib().tdg_conical_rule(dim, order, _ptr(x), _ptr(w))
    return x, w


def facet_vertices(dim: int):
    """Facet-to-vertex map of the unit simplex (lexicographic D-subsets)."""
    return [(0, 1), (0, 2), (1, 2)] if dim == 2 else [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]


def facet_param(dim: int, f: int, chi: np.ndarray) -> np.ndarray:
    """Facet-local points -> element reference coordinates on facet f."""
    verts = np.vstack([np.zeros(dim), np.eye(dim)])
    fv = facet_vertices(dim)[f]
    chi = np.asarray(chi, dtype=np.float64).reshape(-1, dim - 1)
    xi = (1.0 - chi.sum(axis=1))[:, None] * verts[fv[0]]
    for d in range(dim - 1):
        xi = xi + chi[:, d:d + 1] * verts[fv[d + 1]]
    return xi
