"""Shared test inputs: tandem's quadrature rules from the golden fixture and operator cases."""
from __future__ import annotations

import json
from functools import lru_cache
from pathlib import Path

import numpy as np

from tandem_b200 import mesh as M
from tandem_b200.operator import DGOperator, Quadrature
from tandem_b200.scenarios import ElasticityCosine, PoissonSinSin, RandomField

GOLDEN = Path(__file__).resolve().parent / "golden"


@lru_cache(maxsize=None)
def golden(name: str):
    return json.loads((GOLDEN / name).read_text())


def tandem_rule(dim: int, order: int):
    r = golden("quadrature.json")["auto"][f"{dim}:{order}"]
    return np.array(r["points"]).reshape(-1, dim), np.array(r["weights"])


def tandem_quadrature(dim: int, degree: int) -> Quadrature:
    """tandem's volRule / fctRule for MinQuadOrder = 2N + 1 (app/config.h.in:8-11)."""
    order = 2 * degree + 1
    vx, vw = tandem_rule(dim, order)
    fx, fw = tandem_rule(dim - 1, order)
    return Quadrature(vx, vw, fx, fw)


def make_mesh(dim: int, n: int, degree: int, curved: bool = False, bc=M.BC_DIRICHLET, interior_bc=None):
    m = M.square_mesh(n) if dim == 2 else M.cube_mesh(n)
    return M.build(m, degree, boundary_bc=bc, interior_bc=interior_bc,
                   curve=M.box_boundary_surface(0.02) if curved else None)


def material(kind: int, dim: int, X: np.ndarray, variable: bool, seed: int = 1, ell: float = 0.5):
    if kind == 0:
        if variable:
            return (RandomField(dim, seed, ell=ell)(X), None)
        return (np.ones(X.shape[:2]), None)
    if variable:
        return (RandomField(dim, seed, ell=ell)(X), RandomField(dim, seed + 1, ell=ell)(X))
    return (2.0 * np.ones(X.shape[:2]), np.ones(X.shape[:2]))


def scenario(kind: int, dim: int, variable: bool, seed: int = 1, ell: float = 0.5):
    if kind == 0:
        return PoissonSinSin
    if variable:
        return ElasticityCosine(dim, RandomField(dim, seed, ell=ell), RandomField(dim, seed + 1, ell=ell))
    return ElasticityCosine(dim)


def mms_inputs(op, kind: int, dim: int, variable: bool):
    """Material, forcing [E, Q, Nq] and Dirichlet data [F, Q, nq] of the manufactured solution."""
    sc = scenario(kind, dim, variable)
    X, Xf = op.volume_coords(), op.facet_coords()
    if kind == 0:
        c0, c1 = sc.K(X), None
        f = sc.force(X)[:, None, :]
        g = sc.solution(Xf)[:, None, :]
    else:
        c0, c1 = sc.lam(X), sc.mu(X)
        f = np.moveaxis(sc.force(X), -1, 1)
        g = np.moveaxis(sc.solution(Xf), -1, 1)
    return sc, c0, c1, np.ascontiguousarray(f), np.ascontiguousarray(g)


def product_and_oracle(kind: int, dim: int, n: int, degree: int, curved: bool, variable: bool, **mesh_kw):
    from oracle import Oracle
    m = make_mesh(dim, n, degree, curved, **mesh_kw)
    q = tandem_quadrature(dim, degree)
    op = DGOperator(m, degree, kind, q)
    orc = Oracle(m, degree, kind, q)
    c0, c1 = material(kind, dim, op.volume_coords(), variable)
    op.set_material(c0, c1)
    orc.set_material(c0, c1)
    return m, op, orc
