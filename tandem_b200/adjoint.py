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
from .operator import FP64, DGOperator, _check_vec, _stream


class LameProblem:
    """Elasticity solve u(lambda, mu) on a fixed mesh, forcing and boundary data.

    lam, mu: per-element constants [E].  force_Q: [E, D, Nq] or None; bc_q: [F, D, nq] Dirichlet
    and fault slip data or None.  Solves are block-Jacobi CG to `rtol` in `precision`."""

    def __init__(self, op: DGOperator, force_Q=None, bc_q=None, rtol: float = 1e-12, precision: int = FP64,
                 **solve_kw):
        import torch
        if op.kind != 1:
            raise ValueError("LameProblem needs an elasticity operator")
        self.op = op
        self.force_Q = force_Q
        self.bc_q = None if bc_q is None else np.ascontiguousarray(bc_q, dtype=np.float64)
        self._bcq_dev = None if bc_q is None else torch.as_tensor(self.bc_q, device="cuda").contiguous()
        self.rtol = rtol
        self.precision = precision
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
        self.op.bjacobi_setup(self.precision)
        self._theta = key

    def rhs(self):
        import torch
        return torch.as_tensor(self.op.rhs(self.force_Q, self.bc_q), device="cuda")

    def solve(self, b):
        import torch
        x = torch.zeros_like(b)
        st = self.op.solve(b, x, precision=self.precision, rtol=self.rtol, **self.solve_kw)
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
        allocation inside the call.  Meshes up to 4 F + 2 E <= 2^20 (fixed 8 MiB device scratch);
        the FP64 operator data must be resident (an FP64 apply after set_material).  Calls on one
        device must not overlap."""
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
