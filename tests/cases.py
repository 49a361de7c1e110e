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


def mixed_bc_codes(dim: int):
    """Boundary and interior facet codes that exercise every branch of tandem's facet loop
    (Poisson.cpp:591-631, Elasticity.cpp:752-801) on the unit square / cube (n even):
    boundary x=0 Dirichlet, x=1 Natural, y=0 Fault, y=1 None (the element is its own neighbour),
    in 3D also z=0 Dirichlet, z=1 Natural; interior facets on x=0.5 Fault, and a crack of interior
    Natural facets on y=0.5 for x < 0.5 (no flux across it); all other interior facets None."""
    tol = 1e-9

    def on(c, d, v):
        return np.all(np.abs(c[:, :, d] - v) < tol, axis=1)

    def boundary_bc(c):
        out = np.full(c.shape[0], M.BC_DIRICHLET, dtype=np.int32)
        out[on(c, 0, 1.0)] = M.BC_NATURAL
        out[on(c, 1, 0.0)] = M.BC_FAULT
        out[on(c, 1, 1.0)] = M.BC_NONE
        if dim == 3:
            out[on(c, 2, 1.0)] = M.BC_NATURAL
        out[on(c, 0, 0.0)] = M.BC_DIRICHLET
        return out

    def interior_bc(c):
        out = np.full(c.shape[0], M.BC_NONE, dtype=np.int32)
        out[on(c, 0, 0.5)] = M.BC_FAULT
        crack = on(c, 1, 0.5) & np.all(c[:, :, 0] <= 0.5 + tol, axis=1)
        out[crack] = M.BC_NATURAL
        return out

    return boundary_bc, interior_bc


def mixed_bc_mesh(dim: int, n: int, degree: int, curved: bool = False):
    """make_mesh with the facet codes of mixed_bc_codes (n even)."""
    assert n % 2 == 0
    bb, ib = mixed_bc_codes(dim)
    return make_mesh(dim, n, degree, curved, bc=bb, interior_bc=ib)


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


def product_and_oracle(kind: int, dim: int, n: int, degree: int, curved: bool, variable: bool,
                       mixed_bc: bool = False, **mesh_kw):
    from oracle import Oracle
    m = mixed_bc_mesh(dim, n, degree, curved) if mixed_bc else make_mesh(dim, n, degree, curved, **mesh_kw)
    q = tandem_quadrature(dim, degree)
    op = DGOperator(m, degree, kind, q)
    orc = Oracle(m, degree, kind, q)
    c0, c1 = material(kind, dim, op.volume_coords(), variable)
    op.set_material(c0, c1)
    orc.set_material(c0, c1)
    return m, op, orc
