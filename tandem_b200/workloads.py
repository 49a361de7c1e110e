"""Synthetic workloads of the benchmark and the parity tests, built from seeds.

* ``elasticity_cube``: 3D isotropic elasticity, degree N, unit cube n^3 cells x 6 tetrahedra,
  boundary faces curved by a P2 geometry map (amplitude 0.02 sin bump), lambda and mu log-normal
  random fields (mean 1, sigma 0.3, correlation length 0.2, 256 Fourier features), cosine
  manufactured solution with Dirichlet data.
* ``poisson_square``: 2D Poisson, degree N, tandem GenMesh<2> n x n x 2 triangles, K = 1,
  u = sin(pi x) sin(pi y), all-Dirichlet.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import mesh as M
from .operator import DGOperator, ELASTICITY, POISSON, Quadrature
from .scenarios import ElasticityCosine, PoissonSinSin, RandomField


@dataclass
class Workload:
    name: str
    mesh: M.SimplexMesh
    quad: Quadrature
    kind: int
    degree: int
    c0: np.ndarray
    c1: np.ndarray | None
    force: np.ndarray
    bc: np.ndarray
    op: DGOperator


def elasticity_cube(n: int, degree: int, quad: Quadrature, seed: int = 2024, ell: float = 0.2) -> Workload:
    m = M.build(M.cube_mesh(n), degree, curve=M.box_boundary_surface(0.02))
    op = DGOperator(m, degree, ELASTICITY, quad)
    X, Xf = op.volume_coords(), op.facet_coords()
    lam, mu = RandomField(3, seed, ell=ell), RandomField(3, seed + 1, ell=ell)
    sc = ElasticityCosine(3, lam, mu)
    c0, c1 = lam(X), mu(X)
    op.set_material(c0, c1)
    f = np.ascontiguousarray(np.moveaxis(sc.force(X), -1, 1))
    g = np.ascontiguousarray(np.moveaxis(sc.solution(Xf), -1, 1))
    name = f"3D isotropic elasticity p{degree}, unit cube {n}^3 x 6 tets ({m.num_elements:,}), curved P2 boundary, log-normal lambda/mu"
    return Workload(name, m, quad, ELASTICITY, degree, c0, c1, f, g, op)


def poisson_square(n: int, degree: int, quad: Quadrature) -> Workload:
    m = M.build(M.square_mesh(n), degree)
    op = DGOperator(m, degree, POISSON, quad)
    X, Xf = op.volume_coords(), op.facet_coords()
    c0 = PoissonSinSin.K(X)
    op.set_material(c0)
    f = PoissonSinSin.force(X)[:, None, :]
    g = PoissonSinSin.solution(Xf)[:, None, :]
    name = f"2D Poisson SIPG p{degree}, unit square {n}x{n}x2 triangles ({m.num_elements:,}), K=1, sin sin MMS"
    return Workload(name, m, quad, POISSON, degree, c0, None, np.ascontiguousarray(f), np.ascontiguousarray(g), op)
