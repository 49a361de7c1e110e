"""ORACLE -- test infrastructure only (see oracle.cpp).

Python bindings of the CPU restatement of tandem's DG operator and of tandem's own quadrature and
basis sources compiled in place (``oracle/_ref``).  Imported only by tests/, the smoke check and
bench.py's CPU baseline, as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
from math import comb

import numpy as np

from . import build as _build

_p, _i64 = C.c_void_p, C.c_int64
_lib = None
_ref = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = _build.build_oracle()
        L = C.CDLL(str(path))
        sig = {
            "orc_create": (C.c_int, [_p, _p, C.c_int, C.POINTER(_p)]),
            "orc_destroy": (None, [_p]),
            "orc_volume_coords": (None, [_p, _p]),
            "orc_facet_coords": (None, [_p, _p]),
            "orc_facet_normals": (None, [_p, _p]),
            "orc_set_material": (C.c_int, [_p, _p, _p]),
            "orc_material_nodal": (None, [_p, C.c_int, _p]),
            "orc_penalty": (None, [_p, _p]),
            "orc_apply": (None, [_p, _p, _p]),
            "orc_apply_range": (None, [_p, C.c_long, C.c_long, _p, _p]),
            "orc_assemble_diag": (None, [_p, _p]),
            "orc_rhs": (None, [_p, _p, _p, _p]),
            "orc_set_density": (C.c_int, [_p, _p]),
            "orc_apply_inverse_mass": (None, [_p, _p, _p]),
            "orc_cg": (C.c_int, [_p, _p, _p, C.c_double, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
            "orc_error_L2": (C.c_double, [_p, _p, _p]),
            "orc_error_H1_semi": (C.c_double, [_p, _p, _p]),
            "orc_fault_slip_q": (None, [_p, C.c_long, _p, _p, _p, C.c_int, _p, _p]),
            "orc_fault_traction": (None, [_p, C.c_long, _p, _p, _p, C.c_int, _p, _p, _p]),
            "orc_mg_interpolation": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _p]),
            "orc_mg_levels": (C.c_int, [C.c_int, C.c_int, C.c_int, _p]),
            "orc_ref_nodes": (C.c_int, [C.c_int, C.c_int, C.c_int, _p]),
            "orc_ref_basis": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _p, _p]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _lib = L
    return _lib


class Tables:
    """Reference nodes and nodal basis values from the oracle library, with the signatures of
    tandem_b200.refelem's ref_nodes / ref_basis, so that test-side code can build a mesh's geometry
    nodes (tandem_b200.mesh.build(..., tables=Tables)) without loading the product library."""

    @staticmethod
    def ref_nodes(dim: int, degree: int, family: int = 0) -> np.ndarray:
        out = np.zeros((comb(degree + dim, dim), dim))
        lib().orc_ref_nodes(dim, degree, family, out.ctypes.data)
        return out

    @staticmethod
    def ref_basis(dim: int, degree: int, family: int, points: np.ndarray, grad: bool = False):
        if grad:
            raise ValueError("the oracle's tables give basis values only")
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, dim)
        E = np.zeros((comb(degree + dim, dim), pts.shape[0]))
        lib().orc_ref_basis(dim, degree, family, pts.shape[0], pts.ctypes.data, E.ctypes.data)
        return E


def ref_lib() -> C.CDLL | None:
    """tandem's own quadrature/basis code (None where it was never built)."""
    global _ref
    if _ref is None:
        path = _build.build_reference()
        if path is None or not path.exists():
            return None
        L = C.CDLL(str(path))
        L.ref_simplex_rule.restype = C.c_int
        L.ref_simplex_rule.argtypes = [C.c_int, C.c_int, _p, _p]
        L.ref_conical_rule.restype = C.c_int
        L.ref_conical_rule.argtypes = [C.c_int, C.c_int, _p, _p]
        L.ref_gauss_jacobi.restype = C.c_int
        L.ref_gauss_jacobi.argtypes = [C.c_int, C.c_int, C.c_int, _p, _p]
        L.ref_jacobi.restype = C.c_double
        L.ref_jacobi.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double]
        L.ref_dubiner.restype = C.c_double
        L.ref_dubiner.argtypes = [C.c_int, _p, _p]
        L.ref_grad_dubiner.restype = None
        L.ref_grad_dubiner.argtypes = [C.c_int, _p, _p, _p]
        _ref = L
    return _ref


def reference_rule(dim: int, order: int):
    """tandem's simplexQuadratureRule<dim>(order) from the in-place build."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference sources were not built (oracle/_ref missing)")
    n = L.ref_simplex_rule(dim, order, None, None)
    x = np.zeros((n, dim))
    w = np.zeros(n)
    L.ref_simplex_rule(dim, order, x.ctypes.data, w.ctypes.data)
    return x, w


class Oracle:
    """Element-centric CPU operator over the same mesh/quadrature/material inputs as
    tandem_b200.operator.DGOperator."""

    def __init__(self, mesh, degree: int, kind: int, quad):
        from tandem_b200 import _ffi
        L = lib()
        D = mesh.dim
        self.mesh, self.degree, self.kind, self.dim = mesh, degree, kind, D
        c = lambda a, t: np.ascontiguousarray(a, dtype=t)  # noqa: E731
        self._keep = dict(geo=c(mesh.geo_nodes, np.float64), up=c(mesh.facet_up, np.int64),
                          loc=c(mesh.facet_local, np.int32), bc=c(mesh.facet_bc, np.int32),
                          vx=c(quad.vol_x, np.float64), vw=c(quad.vol_w, np.float64),
                          fx=c(quad.fct_x, np.float64), fw=c(quad.fct_w, np.float64))
        k = self._keep
        desc = _ffi.MeshDesc(D, degree, mesh.geo_degree, 0, mesh.num_elements, mesh.num_facets,
                             k["geo"].ctypes.data, k["up"].ctypes.data, k["loc"].ctypes.data, k["bc"].ctypes.data)
        qd = _ffi.Quadrature(len(k["vw"]), len(k["fw"]), k["vx"].ctypes.data, k["vw"].ctypes.data,
                             k["fx"].ctypes.data, k["fw"].ctypes.data)
        h = C.c_void_p()
        if L.orc_create(C.byref(desc), C.byref(qd), kind, C.byref(h)) != 0:
            raise RuntimeError("oracle construction failed")
        self._h = h
        self.Q = 1 if kind == 0 else D
        self.nbf = comb(degree + D, D)
        self.bs = self.nbf * self.Q
        self.E, self.F = mesh.num_elements, mesh.num_facets
        self.Nq, self.nq = len(k["vw"]), len(k["fw"])

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().orc_destroy(h)
            self._h = None

    @property
    def ndof(self) -> int:
        return self.E * self.bs

    def volume_coords(self):
        out = np.zeros((self.E, self.Nq, self.dim))
        lib().orc_volume_coords(self._h, out.ctypes.data)
        return out

    def facet_coords(self):
        out = np.zeros((self.F, self.nq, self.dim))
        lib().orc_facet_coords(self._h, out.ctypes.data)
        return out

    def facet_normals(self):
        out = np.zeros((self.F, self.nq, self.dim))
        lib().orc_facet_normals(self._h, out.ctypes.data)
        return out

    def set_material(self, c0_Q, c1_Q=None):
        a = np.ascontiguousarray(c0_Q, dtype=np.float64).reshape(self.E, self.Nq)
        b = a if c1_Q is None else np.ascontiguousarray(c1_Q, dtype=np.float64).reshape(self.E, self.Nq)
        self._mat = (a, b)
        lib().orc_set_material(self._h, a.ctypes.data, b.ctypes.data)

    def material_nodal(self, c: int):
        out = np.zeros((self.E, self.nbf))
        lib().orc_material_nodal(self._h, c, out.ctypes.data)
        return out

    def penalty(self):
        out = np.zeros(self.F)
        lib().orc_penalty(self._h, out.ctypes.data)
        return out

    def apply(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        lib().orc_apply(self._h, x.ctypes.data, y.ctypes.data)
        return y

    def apply_range(self, e0: int, e1: int, x: np.ndarray, y: np.ndarray) -> None:
        lib().orc_apply_range(self._h, e0, e1, x.ctypes.data, y.ctypes.data)

    def assemble_diag(self) -> np.ndarray:
        out = np.zeros((self.E, self.bs, self.bs))
        lib().orc_assemble_diag(self._h, out.ctypes.data)
        return np.ascontiguousarray(out.transpose(0, 2, 1))  # [e, row, col]

    def set_density(self, rho_Q):
        """Elasticity density at the volume points [E, Nq] (default 1)."""
        r = np.ascontiguousarray(rho_Q, dtype=np.float64).reshape(self.E, self.Nq)
        lib().orc_set_density(self._h, r.ctypes.data)

    def apply_inverse_mass(self, x: np.ndarray) -> np.ndarray:
        """-1/rho weighted inverse mass of Elasticity::wave_rhs applied to x."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.ndof)
        lib().orc_apply_inverse_mass(self._h, x.ctypes.data, y.ctypes.data)
        return y

    def rhs(self, force_Q=None, bc_q=None) -> np.ndarray:
        b = np.zeros(self.ndof)
        f = None if force_Q is None else np.ascontiguousarray(force_Q, dtype=np.float64)
        g = None if bc_q is None else np.ascontiguousarray(bc_q, dtype=np.float64)
        lib().orc_rhs(self._h, None if f is None else f.ctypes.data, None if g is None else g.ctypes.data,
                      b.ctypes.data)
        return b

    def cg(self, b: np.ndarray, rtol: float = 1e-10, maxit: int = 20000, x0=None):
        x = np.zeros(self.ndof) if x0 is None else np.array(x0, dtype=np.float64)
        it, rel = C.c_int(0), C.c_double(0.0)
        rc = lib().orc_cg(self._h, np.ascontiguousarray(b).ctypes.data, x.ctypes.data, rtol, maxit,
                          C.byref(it), C.byref(rel))
        return x, dict(iterations=it.value, rel_residual=rel.value, converged=rc == 0)

    def fault_basis(self):
        """tandem's fault space (nodal warp & blend of degree N on the facet) at the facet points."""
        from tandem_b200.refelem import WARP_BLEND, ref_basis
        fx = np.asarray(self._keep["fx"]).reshape(-1, self.dim - 1)
        return np.ascontiguousarray(ref_basis(self.dim - 1, self.degree, WARP_BLEND, fx))

    def fault_slip_q(self, facets, ref_normal, slip):
        e = self.fault_basis()
        f = np.ascontiguousarray(facets, dtype=np.int64)
        r = np.ascontiguousarray(ref_normal, dtype=np.float64)
        sl = np.ascontiguousarray(slip, dtype=np.float64)
        out = np.zeros((self.F, 1, self.nq))
        lib().orc_fault_slip_q(self._h, len(f), f.ctypes.data, r.ctypes.data, e.ctypes.data, e.shape[0],
                               sl.ctypes.data, out.ctypes.data)
        return out

    def fault_traction(self, facets, ref_normal, u, slip):
        e = self.fault_basis()
        f = np.ascontiguousarray(facets, dtype=np.int64)
        r = np.ascontiguousarray(ref_normal, dtype=np.float64)
        sl = np.ascontiguousarray(slip, dtype=np.float64)
        uu = np.ascontiguousarray(u, dtype=np.float64)
        out = np.zeros((len(f), e.shape[0]))
        lib().orc_fault_traction(self._h, len(f), f.ctypes.data, r.ctypes.data, e.ctypes.data, e.shape[0],
                                 uu.ctypes.data, sl.ctypes.data, out.ctypes.data)
        return out

    def error_L2(self, x: np.ndarray, ref_Q: np.ndarray) -> float:
        r = np.ascontiguousarray(ref_Q, dtype=np.float64)
        return lib().orc_error_L2(self._h, np.ascontiguousarray(x).ctypes.data, r.ctypes.data)

    def error_H1_semi(self, x: np.ndarray, refgrad_Q: np.ndarray) -> float:
        r = np.ascontiguousarray(refgrad_Q, dtype=np.float64)
        return lib().orc_error_H1_semi(self._h, np.ascontiguousarray(x).ctypes.data, r.ctypes.data)


# ---- p-multigrid restated (tandem's PCMG configuration) ---------------------------------------------

def mg_interpolation(dim: int, kind: int, n_to: int, n_from: int) -> np.ndarray:
    """One component's interpolation block [Nbf(n_to), Nbf(n_from)] as tandem assembles it
    (NodalInterpolation.cpp:8-36 / ModalInterpolation.h:31-45)."""
    from math import comb
    out = np.zeros((comb(n_to + dim, dim), comb(n_from + dim, dim)))
    if lib().orc_mg_interpolation(dim, kind, n_to, n_from, out.ctypes.data) != 0:
        raise ValueError("bad interpolation degrees")
    return out


def mg_levels(strategy: int, coarse: int, degree: int) -> list[int]:
    """MGConfig::levels (app/common/MGConfig.cpp:11-41), coarsest first."""
    out = (C.c_int * 32)()
    n = lib().orc_mg_levels(strategy, coarse, degree, out)
    if n < 0:
        raise ValueError("bad strategy")
    return list(out[:n])


def element_interpolation(E: int, Q: int, I: np.ndarray) -> np.ndarray:
    """Dense block-diagonal interpolation of E elements (tandem's InterpolationOperator::assemble,
    src/form/InterpolationOperator.h:28-49): I(k + p N1, l + p N2) per element and component."""
    return np.kron(np.eye(E), np.kron(np.eye(Q), I))


class DenseMultigrid:
    """The V-cycle of PETSc's PCMG as tandem configures it (app/common/PetscLinearSolver.cpp:53-114,
    examples/options/mg_cheby.cfg) on dense matrices: Galerkin coarse operators A_l = P^T A_{l+1} P,
    Chebyshev smoothing with point Jacobi on [lo, hi] x lambda_max (Saad, Iterative Methods, Alg.
    12.1), the same number of steps before and after the coarse correction, and an exact solve on
    the coarsest level.  lambda_max per smoothed level is given (the product's estimates), so the
    restatement and the device V-cycle apply the same polynomials."""

    def __init__(self, A: np.ndarray, P: list[np.ndarray], lmax: list[float], smooth_its: int = 10,
                 esteig: tuple[float, float] = (0.01, 1.1)):
        self.P = P  # P[l]: level l -> level l + 1
        self.A = [None] * len(P) + [A]
        for l in range(len(P) - 1, -1, -1):
            self.A[l] = P[l].T @ self.A[l + 1] @ P[l]
        self.lmax, self.its, self.esteig = lmax, smooth_its, esteig

    def smooth(self, l: int, b: np.ndarray, x: np.ndarray | None) -> np.ndarray:
        A = self.A[l]
        dinv = 1.0 / np.diag(A)
        emax, emin = self.esteig[1] * self.lmax[l], self.esteig[0] * self.lmax[l]
        theta, delta = 0.5 * (emax + emin), 0.5 * (emax - emin)
        sigma = theta / delta
        rho = 1.0 / sigma
        r = b.copy() if x is None else b - A @ x
        d = dinv * r / theta
        x = d.copy() if x is None else x + d
        for _ in range(1, self.its):
            r = r - A @ d
            rho1 = 1.0 / (2.0 * sigma - rho)
            d = rho1 * rho * d + 2.0 * rho1 / delta * dinv * r
            x = x + d
            rho = rho1
        return x

    def vcycle(self, b: np.ndarray, l: int | None = None) -> np.ndarray:
        l = len(self.A) - 1 if l is None else l
        if l == 0:
            return np.linalg.solve(self.A[0], b)
        x = self.smooth(l, b, None)
        r = b - self.A[l] @ x
        x = x + self.P[l - 1] @ self.vcycle(self.P[l - 1].T @ r, l - 1)
        return self.smooth(l, b, x)
