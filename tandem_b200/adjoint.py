"""Gradients of functionals of the elastic displacement with respect to per-element constant Lame
parameters, by the adjoint method (tandem itself solves forward problems only; this wraps its
elasticity operator, app/pde/Elasticity.cpp, as a differentiable map theta -> u).

For A(theta) u = b(theta) with symmetric A (SIPG with epsilon = -1):

    dJ/dtheta_e = p^T db/dtheta_e - p^T dA/dtheta_e u,   A p = dJ/du,

one forward solve, one adjoint solve with the same operator and preconditioner, and one
gradient kernel launch (tdg_adjoint_lame_gradient) that contracts the element and facet terms of
element e with u and p.  `LameSolve` exposes the map as a torch.autograd.Function, so any torch
loss of u back-propagates to (lambda, mu)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi
from .operator import FP32, FP64, DGOperator, _check_vec, _stream


class LameProblem:
    """Elasticity solve u(lambda, mu) on a fixed mesh, forcing and boundary data.

    lam, mu: per-element constants [E].  force_Q: [E, D, Nq] or None; bc_q: [F, D, nq] Dirichlet
    and fault slip data or None.  Solves are CG to `rtol` in `precision`, preconditioned by block
    Jacobi or (preconditioner="mg") by the p-multigrid V-cycle, rebuilt whenever the parameters
    change."""

    def __init__(self, op: DGOperator, force_Q=None, bc_q=None, rtol: float = 1e-12, precision: int = FP64,
                 preconditioner: str = "bjacobi", **solve_kw):
        import torch
        if op.kind != 1:
            raise ValueError("LameProblem needs an elasticity operator")
        self.op = op
        self.force_Q = force_Q
        self.bc_q = None if bc_q is None else np.ascontiguousarray(bc_q, dtype=np.float64)
        self._bcq_dev = None if bc_q is None else torch.as_tensor(self.bc_q, device="cuda").contiguous()
        self.rtol = rtol
        self.precision = precision
        self.pc_precision = FP64 if precision != FP32 else FP32
        if preconditioner not in ("bjacobi", "mg") or (preconditioner == "mg" and precision == FP32):
            raise ValueError("preconditioner: 'bjacobi', or 'mg' with FP64 / MIXED solves")
        self.preconditioner = preconditioner
        self.solve_kw = solve_kw
        self._theta = None
        self.last_stats: list[dict] = []

    def set_parameters(self, lam, mu) -> None:
        lam = np.asarray(lam, dtype=np.float64).reshape(-1)
        mu = np.asarray(mu, dtype=np.float64).reshape(-1)
        if lam.shape != (self.op.E,) or mu.shape != (self.op.E,):
            raise ValueError(f"expected per-element parameters of shape ({self.op.E},)")
        key = (lam.tobytes(), mu.tobytes())
        if self._theta == key:
            return
        ones = np.ones((1, self.op.Nq))
        self.op.set_material(lam[:, None] * ones, mu[:, None] * ones)
        if self.preconditioner == "mg":
            self.op.mg_setup(smooth_precision=self.precision)
            self.op.set_preconditioner("mg")
        else:
            self.op.set_preconditioner("bjacobi")
            self.op.bjacobi_setup(self.pc_precision)
        self._theta = key

    def rhs(self):
        import torch
        return torch.as_tensor(self.op.rhs(self.force_Q, self.bc_q), device="cuda")

    def solve(self, b):
        """Solves to `rtol`; a problem whose attainable FP64 accuracy lies above rtol returns the
        best iterate (its residual is in last_stats) instead of raising."""
        import torch
        x = torch.zeros_like(b)
        st = self.op.solve(b, x, precision=self.precision, rtol=self.rtol, check=False, **self.solve_kw)
        self.last_stats.append(st)
        return x

    def forward(self, lam, mu):
        """u(lam, mu) as a CUDA float64 tensor [ndof]."""
        self.set_parameters(lam, mu)
        return self.solve(self.rhs())

    def gradient(self, u, p, stream=None):
        """[E, 2] = (dJ/dlam_e, dJ/dmu_e) for state u and adjoint p (both at the current parameters)."""
        import torch
        _check_vec(u, FP64, self.op.ndof)
        _check_vec(p, FP64, self.op.ndof)
        g = torch.empty(self.op.E, 2, dtype=torch.float64, device="cuda")
        bcq = None if self._bcq_dev is None else C.c_void_p(self._bcq_dev.data_ptr())
        _ffi.check(_ffi.lib().tdg_adjoint_lame_gradient(self.op._h, C.c_void_p(u.data_ptr()),
                                                        C.c_void_p(p.data_ptr()), bcq,
                                                        C.c_void_p(g.data_ptr()), _stream(stream)))
        return g

    def gradient_noalloc(self, u, p, grad, stream=None):
        """Allocation-free gradient into the caller's grad [E, 2] (CUDA float64): no device or host
        allocation inside a successful call, for loops that cannot allocate device memory (their
        process's caching pool holds it).  Meshes up to 4 F + 2 E <= 2^20 (fixed 8 MiB device
        scratch); the FP64 operator data must be resident (an FP64 apply after set_material, which
        also prepares the scratch and the kernel).  Calls on one device must not overlap."""
        _check_vec(u, FP64, self.op.ndof)
        _check_vec(p, FP64, self.op.ndof)
        _check_vec(grad, FP64, 2 * self.op.E)
        bcq = None if self._bcq_dev is None else C.c_void_p(self._bcq_dev.data_ptr())
        _ffi.check(_ffi.lib().tdg_adjoint_lame_gradient_noalloc(self.op._h, C.c_void_p(u.data_ptr()),
                                                                C.c_void_p(p.data_ptr()), bcq,
                                                                C.c_void_p(grad.data_ptr()), _stream(stream)))


def _make_function():
    import torch

    class LameSolve(torch.autograd.Function):
        """u = LameSolve.apply(lam, mu, problem): differentiable in lam and mu [E] (float64)."""

        @staticmethod
        def forward(ctx, lam, mu, problem: LameProblem):
            u = problem.forward(lam.detach().cpu().numpy(), mu.detach().cpu().numpy())
            ctx.problem = problem
            ctx.theta = (lam.detach().cpu().numpy().copy(), mu.detach().cpu().numpy().copy())
            ctx.devices = (lam.device, mu.device)
            ctx.save_for_backward(u)
            return u

        @staticmethod
        def backward(ctx, grad_u):
            (u,) = ctx.saved_tensors
            pb = ctx.problem
            pb.set_parameters(*ctx.theta)
            p = pb.solve(grad_u.contiguous().to(torch.float64))
            g = pb.gradient(u, p)
            return g[:, 0].to(ctx.devices[0]), g[:, 1].to(ctx.devices[1]), None

    return LameSolve


class _Lazy:
    fn = None


def lame_solve(lam, mu, problem: LameProblem):
    """Differentiable u(lam, mu); lam, mu: torch float64 tensors [E]."""
    if _Lazy.fn is None:
        _Lazy.fn = _make_function()
    return _Lazy.fn.apply(lam, mu, problem)


class PointObservation:
    """Displacement at given points, P u -> [npts, Q], for points inside affine elements (the
    interior of a mesh whose curving only touches boundary elements).  Each point is located by its
    barycentric coordinates in the element's vertex order (the order of the reference map), and the
    element's nodal basis is evaluated at the reference coordinates.  `apply` is a torch gather, so
    autograd supplies P^T."""

    def __init__(self, mesh, degree: int, points, Q: int | None = None, chunk: int = 32, device: str = "cuda"):
        import torch
        from . import refelem
        pts = np.ascontiguousarray(points, dtype=np.float64)
        D = mesh.dim
        Q = D if Q is None else Q
        V, El = mesh.vertices, mesh.elements
        v0 = V[El[:, 0]]
        T = np.transpose(V[El[:, 1:]] - v0[:, None, :], (0, 2, 1))  # columns = edges from v0
        Tinv = np.linalg.inv(T)
        elem = np.full(len(pts), -1, dtype=np.int64)
        xi = np.zeros((len(pts), D))
        for s in range(0, len(pts), chunk):
            p = pts[s:s + chunk]
            loc = np.einsum("eij,pej->pei", Tinv, p[:, None, :] - v0[None, :, :])
            bary = np.concatenate([1.0 - loc.sum(axis=2, keepdims=True), loc], axis=2)
            inside = np.all(bary >= -1e-12, axis=2)
            for i in range(len(p)):
                hit = np.nonzero(inside[i])[0]
                if len(hit) == 0:
                    raise ValueError(f"point {pts[s + i]} is outside the mesh")
                elem[s + i] = hit[0]
                xi[s + i] = loc[i, hit[0]]
        E = refelem.ref_basis(D, degree, refelem.WARP_BLEND, xi)  # [Nbf][npts]
        nbf = E.shape[0]
        bs = nbf * Q
        k = np.arange(nbf)
        idx = elem[:, None, None] * bs + k[None, None, :] + nbf * np.arange(Q)[None, :, None]
        self.elements, self.xi = elem, xi
        self.index = torch.as_tensor(idx.reshape(len(pts), -1), device=device)
        self.weight = torch.as_tensor(np.ascontiguousarray(E.T), device=device)  # [npts, Nbf]
        self.npts, self.Q, self.nbf = len(pts), Q, nbf

    def apply(self, u):
        g = u[self.index].view(self.npts, self.Q, self.nbf)
        return (g * self.weight[:, None, :]).sum(dim=2)
