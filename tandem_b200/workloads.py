"""Synthetic workloads of the benchmark and the parity tests, built from seeds.

* ``elasticity_cube``: 3D isotropic elasticity, degree N, unit cube n^3 cells x 6 tetrahedra,
  boundary faces curved by a P2 geometry map (amplitude 0.02 sin bump), lambda and mu log-normal
  random fields (mean 1, sigma 0.3, correlation length 0.2, 256 Fourier features), cosine
  manufactured solution with Dirichlet data.
* ``poisson_square``: 2D Poisson, degree N, tandem GenMesh<2> n x n x 2 triangles, K = 1,
  u = sin(pi x) sin(pi y), all-Dirichlet.
* ``uneven_batch``: `count` independent 2D elasticity problems, degree N, on unit squares with
  P2-curved boundaries whose element counts are log-uniform in [lo, hi] (seeded), each with its
  own log-normal random lambda / mu (as above) and a random-Fourier-feature body force,
  homogeneous Dirichlet data; held as one block-diagonal operator over the mesh union.
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


@dataclass
class Batch:
    name: str
    mesh: M.SimplexMesh
    quad: Quadrature
    degree: int
    elem_offsets: np.ndarray
    sizes: np.ndarray
    force: np.ndarray
    bc: np.ndarray
    op: DGOperator


def uneven_batch_cells(count: int, seed: int = 7, lo: int = 1000, hi: int = 40000) -> np.ndarray:
    """Cells per direction of each problem's n x n x 2 mesh (element counts log-uniform in [lo, hi])."""
    rng = np.random.Generator(np.random.PCG64(seed))
    target = np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))
    return np.maximum(2, np.rint(np.sqrt(target / 2.0))).astype(int)


def uneven_batch(count: int, degree: int, quad: Quadrature, seed: int = 7, lo: int = 1000, hi: int = 40000,
                 ell: float = 0.2, problems=None) -> Batch:
    """The batch, or only the problems listed in `problems` (a rank's share of it; every problem's
    mesh, material and force depend on its index alone)."""
    cells = uneven_batch_cells(count, seed, lo, hi)
    which = list(range(count)) if problems is None else [int(i) for i in problems]
    meshes = [M.build(M.square_mesh(int(cells[i])), degree, curve=M.box_boundary_surface(0.02)) for i in which]
    um, eoff = M.union(meshes)
    op = DGOperator(um, degree, ELASTICITY, quad)
    X = op.volume_coords()
    lam = np.empty(X.shape[:2])
    mu = np.empty(X.shape[:2])
    force = np.empty((op.E, 2, op.Nq))
    for j, i in enumerate(which):
        sl = slice(eoff[j], eoff[j + 1])
        s = seed * 1000 + 10 * i
        lam[sl] = RandomField(2, s + 1, ell=ell)(X[sl])
        mu[sl] = RandomField(2, s + 2, ell=ell)(X[sl])
        force[sl, 0] = RandomField(2, s + 3, ell=ell, mean=0.0, sigma=1.0, lognormal=False)(X[sl])
        force[sl, 1] = RandomField(2, s + 4, ell=ell, mean=0.0, sigma=1.0, lognormal=False)(X[sl])
    op.set_material(lam, mu)
    bc = np.zeros((op.F, 2, op.nq))
    sizes = np.diff(eoff)
    name = (f"{len(which)} independent 2D elasticity problems p{degree}, curved P2 unit squares, "
            f"{int(sizes.min()):,}-{int(sizes.max()):,} triangles each ({op.E:,} total), log-normal lambda/mu, "
            f"RFF body force, zero Dirichlet")
    return Batch(name, um, quad, degree, eoff, sizes, np.ascontiguousarray(force), bc, op)
