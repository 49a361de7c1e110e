"""Closed-form scenarios (coefficients, manufactured solutions, forcing) evaluated at the
quadrature-point coordinates the operator exposes -- the role tandem's Lua scenarios play
(app/common/Scenario.h:37-78).

* ``PoissonSinSin``: -div(K grad u) = f with K = 1, u = sin(pi x) sin(pi y) (2D), f = 2 pi^2 u.
* ``RandomField``: smooth log-normal field mean exp(sigma Z - sigma^2 / 2) (or the Gaussian field
  mean + sigma Z), Z a unit-variance Gaussian random field with Gaussian covariance of length ell
  realised by M random Fourier features from a seed (closed form, so gradients are exact).
* ``ElasticityCosine``: isotropic elasticity with variable lambda, mu and the cosine manufactured
  solution of tandem's examples/elasticity/3d/cosine.lua, u = (cos pi x cos pi y, 0,
  cos pi x cos pi z) (2D: (cos pi x cos pi y, 0)); f = -div sigma(u) with
  sigma = lam tr(eps) I + 2 mu eps, i.e.
  f = -[(div u) grad lam + lam grad div u + 2 eps grad mu + mu (lap u + grad div u)].
"""
from __future__ import annotations

import numpy as np

PI = np.pi


class PoissonSinSin:
    dim = 2

    @staticmethod
    def K(x):
        return np.ones(x.shape[:-1])

    @staticmethod
    def solution(x):
        return np.sin(PI * x[..., 0]) * np.sin(PI * x[..., 1])

    @staticmethod
    def gradient(x):
        s0, s1 = np.sin(PI * x[..., 0]), np.sin(PI * x[..., 1])
        c0, c1 = np.cos(PI * x[..., 0]), np.cos(PI * x[..., 1])
        return np.stack([PI * c0 * s1, PI * s0 * c1], axis=-1)

    @classmethod
    def force(cls, x):
        return 2.0 * PI * PI * cls.solution(x)


class RandomField:
    def __init__(self, dim: int, seed: int, ell: float = 0.2, sigma: float = 0.3, features: int = 256,
                 mean: float = 1.0, lognormal: bool = True):
        rng = np.random.Generator(np.random.PCG64(seed))
        self.omega = rng.normal(0.0, 1.0 / ell, size=(features, dim))
        self.phase = rng.uniform(0.0, 2.0 * PI, size=features)
        self.amp = np.sqrt(2.0 / features)
        self.sigma, self.mean, self.lognormal = sigma, mean, lognormal

    CHUNK = 1 << 18  # points per block (bounds the [points, features] temporaries)

    def value_and_gradient(self, x, grad: bool = True):
        """Field values (and gradients) at points x [..., dim], evaluated with torch (on the GPU
        when one is present, else on all CPU cores) in float64."""
        import torch
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        shape = np.shape(x)
        pts = torch.as_tensor(np.asarray(x, dtype=np.float64).reshape(-1, shape[-1]), device=dev)
        om = torch.as_tensor(self.omega, device=dev)
        ph = torch.as_tensor(self.phase, device=dev)
        z = torch.empty(pts.shape[0], dtype=torch.float64, device=dev)
        dz = torch.empty_like(pts) if grad else None
        for s in range(0, pts.shape[0], self.CHUNK):
            arg = pts[s:s + self.CHUNK] @ om.T + ph
            z[s:s + self.CHUNK] = self.amp * torch.cos(arg).sum(dim=1)
            if grad:
                dz[s:s + self.CHUNK] = -self.amp * (torch.sin(arg) @ om)
        if self.lognormal:
            v = self.mean * torch.exp(self.sigma * z - 0.5 * self.sigma ** 2)
            scale = self.sigma * v
        else:  # Gaussian field mean + sigma Z
            v = self.mean + self.sigma * z
            scale = torch.full_like(z, self.sigma)
        val = v.cpu().numpy().reshape(shape[:-1])
        if not grad:
            return val, None
        g = (scale[:, None] * dz).cpu().numpy().reshape(shape)
        return val, g

    def __call__(self, x):
        return self.value_and_gradient(x, grad=False)[0]

    def gradient(self, x):
        return self.value_and_gradient(x)[1]


class ConstantField:
    def __init__(self, value: float):
        self.value = value

    def __call__(self, x):
        return np.full(x.shape[:-1], self.value)

    def gradient(self, x):
        return np.zeros(x.shape)

    def value_and_gradient(self, x, grad: bool = True):
        return self(x), (self.gradient(x) if grad else None)


class ElasticityCosine:
    def __init__(self, dim: int, lam=None, mu=None):
        self.dim = dim
        self.lam = lam if lam is not None else ConstantField(2.0)
        self.mu = mu if mu is not None else ConstantField(1.0)

    def solution(self, x):
        cx, cy = np.cos(PI * x[..., 0]), np.cos(PI * x[..., 1])
        if self.dim == 2:
            return np.stack([cx * cy, np.zeros_like(cx)], axis=-1)
        cz = np.cos(PI * x[..., 2])
        return np.stack([cx * cy, np.zeros_like(cx), cx * cz], axis=-1)

    def gradient(self, x):
        """J[..., i, d] = d u_i / d x_d."""
        sx, sy = np.sin(PI * x[..., 0]), np.sin(PI * x[..., 1])
        cx, cy = np.cos(PI * x[..., 0]), np.cos(PI * x[..., 1])
        J = np.zeros(x.shape[:-1] + (self.dim, self.dim))
        J[..., 0, 0] = -PI * sx * cy
        J[..., 0, 1] = -PI * cx * sy
        if self.dim == 3:
            sz, cz = np.sin(PI * x[..., 2]), np.cos(PI * x[..., 2])
            J[..., 2, 0] = -PI * sx * cz
            J[..., 2, 2] = -PI * cx * sz
        return J

    def force(self, x):
        D = self.dim
        sx, sy = np.sin(PI * x[..., 0]), np.sin(PI * x[..., 1])
        cx, cy = np.cos(PI * x[..., 0]), np.cos(PI * x[..., 1])
        P2 = PI * PI
        J = self.gradient(x)
        div = np.trace(J, axis1=-2, axis2=-1)
        gdiv = np.zeros(x.shape[:-1] + (D,))
        lap = np.zeros(x.shape[:-1] + (D,))
        # u1 = cx cy
        gdiv[..., 0] += -P2 * cx * cy
        gdiv[..., 1] += P2 * sx * sy
        lap[..., 0] = -2.0 * P2 * cx * cy
        if D == 3:
            sz, cz = np.sin(PI * x[..., 2]), np.cos(PI * x[..., 2])
            # u3 = cx cz: d/dx(-pi cx sz) = pi^2 sx sz, d/dz(...) = -pi^2 cx cz
            gdiv[..., 0] += P2 * sx * sz
            gdiv[..., 2] += -P2 * cx * cz
            lap[..., 2] = -2.0 * P2 * cx * cz
        lam, glam = self.lam.value_and_gradient(x)
        mu, gmu = self.mu.value_and_gradient(x)
        eps = 0.5 * (J + np.swapaxes(J, -1, -2))
        divsig = (div[..., None] * glam + lam[..., None] * gdiv + 2.0 * np.einsum("...ij,...j->...i", eps, gmu)
                  + mu[..., None] * (lap + gdiv))
        return -divsig
