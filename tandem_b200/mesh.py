"""Simplex meshes, topology and curvilinear geometry nodes.

Generators:
  * ``square_mesh`` -- tandem's ``GenMesh<2>`` tessellation of a structured square: vertex ids
    flattened x-fastest (src/util/MultiIndex.h:22-29), each cell split into two triangles with the
    diagonal alternating by cell parity (src/mesh/GenMesh.cpp:20-32,118-121);
  * ``cube_mesh`` -- unit cube, each cell split into 6 tetrahedra (Kuhn / Freudenthal split; tandem's
    own GenMesh<3> uses 5, src/mesh/GenMesh.cpp:34-52);
  * ``graded_fault_mesh`` -- 2D antiplane domain graded toward a planar dipping fault.
Element vertices are sorted by global id, which is what makes the facet quadrature points of the
two sides of a facet coincide (src/mesh/Simplex.h:15-36).

``topology`` builds tandem's FacetInfo arrays (up, localNo, bc; src/form/DGOperatorTopo.cpp:46-85)
and ``geometry_nodes`` the degree-N warp & blend geometry nodes of Curvilinear, optionally from P2
element nodes (src/geometry/Curvilinear.cpp:59-112).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from itertools import permutations
from typing import Callable

import numpy as np

from .refelem import EQUIDISTANT, WARP_BLEND, facet_vertices, ref_basis, ref_nodes

BC_NONE, BC_NATURAL, BC_FAULT, BC_DIRICHLET = 0, 1, 3, 5

# VTK edge order of P2 nodes (src/basis/NumberingConvention.h)
EDGES = {2: [(0, 1), (1, 2), (2, 0)], 3: [(0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)]}


@dataclass
class SimplexMesh:
    dim: int
    vertices: np.ndarray  # [V, D]
    elements: np.ndarray  # [E, D+1] int64, sorted
    facets: np.ndarray = None  # [F, D] vertex ids
    facet_up: np.ndarray = None  # [F, 2] int64
    facet_local: np.ndarray = None  # [F, 2] int32
    facet_bc: np.ndarray = None  # [F] int32
    geo_degree: int = 1
    geo_nodes: np.ndarray = None  # [E, Ngeo, D]
    p2_nodes: np.ndarray = None  # [E, nP2, D] (curved meshes)
    info: dict = field(default_factory=dict)

    @property
    def num_elements(self) -> int:
        return self.elements.shape[0]

    @property
    def num_facets(self) -> int:
        return self.facets.shape[0]


def square_mesh(n: int, extent=(1.0, 1.0)) -> SimplexMesh:
    """tandem GenMesh<2>({n, n}) on [0, extent]^2."""
    np1 = n + 1
    iy, ix = np.meshgrid(np.arange(np1), np.arange(np1), indexing="ij")
    verts = np.stack([ix.ravel() * extent[0] / n, iy.ravel() * extent[1] / n], axis=1)
    ey, ex = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    ex, ey = ex.ravel(), ey.ravel()  # cube index flattened x-fastest
    g = lambda dx, dy: (ex + dx) + np1 * (ey + dy)  # noqa: E731
    v00, v01, v10, v11 = g(0, 0), g(1, 0), g(0, 1), g(1, 1)  # bit 0 -> x, bit 1 -> y
    odd = ((ex % 2) ^ (ey % 2)).astype(bool)
    t0 = np.where(odd[:, None], np.stack([v00, v01, v11], 1), np.stack([v00, v01, v10], 1))
    t1 = np.where(odd[:, None], np.stack([v00, v10, v11], 1), np.stack([v01, v10, v11], 1))
    el = np.empty((2 * ex.size, 3), dtype=np.int64)
    el[0::2] = t0
    el[1::2] = t1
    return SimplexMesh(2, verts, np.sort(el, axis=1))


def cube_mesh(n: int) -> SimplexMesh:
    """Unit cube, n^3 cells, 6 Kuhn tetrahedra per cell (all sharing the 000-111 diagonal)."""
    np1 = n + 1
    iz, iy, ix = np.meshgrid(np.arange(np1), np.arange(np1), np.arange(np1), indexing="ij")
    verts = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1) / n
    ez, ey, ex = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
    unit = np.eye(3, dtype=np.int64)
    tets = []
    for perm in permutations(range(3)):
        pts = [np.zeros(3, dtype=np.int64)]
        for a in perm:
            pts.append(pts[-1] + unit[a])
        tets.append(pts)
    el = np.empty((ex.size * 6, 4), dtype=np.int64)
    for t, pts in enumerate(tets):
        cols = [(ex + p[0]) + np1 * ((ey + p[1]) + np1 * (ez + p[2])) for p in pts]
        el[t::6] = np.stack(cols, axis=1)
    return SimplexMesh(3, verts, np.sort(el, axis=1))


def _graded(h0: float, length: float, ratio: float) -> np.ndarray:
    """Offsets 0 < d_1 < ... = length with first step h0 and geometric growth `ratio`."""
    d, h, out = 0.0, h0, []
    while d + h < length - 0.5 * h:
        d += h
        out.append(d)
        h *= ratio
    out.append(length)
    return np.array(out)


def graded_fault_mesh(num_fault_facets: int = 256, fault_length: float = 12.8, dip_deg: float = 60.0,
                      width: float = 40.0, depth: float = 20.0, ratio: float = 1.07):
    """2D antiplane domain (km) graded toward a planar dipping fault.

    The domain is the parallelogram {x = xi - s cot(dip), y = s}, xi in [-width/2, width/2],
    s in [-depth, 0]: its slanted sides follow the fault, which is the grid line xi = 0 from the
    free surface (y = 0) down to the fault tip.  Along the fault the grid spacing is
    fault_length / num_fault_facets; away from it cells grow geometrically by `ratio`.
    Boundary conditions: free surface Natural, the other three sides Dirichlet; the interior facets
    on xi = 0 above the tip are Fault facets (ordered by depth)."""
    theta = np.deg2rad(dip_deg)
    h_f = fault_length / num_fault_facets
    tip = -fault_length * np.sin(theta)
    ds = h_f * np.sin(theta)
    s_fault = np.linspace(tip, 0.0, num_fault_facets + 1)
    s_below = tip - _graded(ds, depth + tip, ratio)
    s = np.concatenate([s_below[::-1], s_fault])
    xi_r = _graded(h_f, 0.5 * width, ratio)
    xi = np.concatenate([-xi_r[::-1], [0.0], xi_r])
    nx, ns = xi.size, s.size
    S, XI = np.meshgrid(s, xi, indexing="ij")  # vertex (j, i) -> id i + nx * j
    X = XI - S / np.tan(theta)  # s <= 0: the fault dips toward +x
    verts = np.stack([X.ravel(), S.ravel()], axis=1)
    ci, cj = np.meshgrid(np.arange(nx - 1), np.arange(ns - 1), indexing="xy")
    ci, cj = ci.ravel(), cj.ravel()
    v00 = ci + nx * cj
    v01, v10, v11 = v00 + 1, v00 + nx, v00 + nx + 1
    odd = ((ci % 2) ^ (cj % 2)).astype(bool)
    t0 = np.where(odd[:, None], np.stack([v00, v01, v11], 1), np.stack([v00, v01, v10], 1))
    t1 = np.where(odd[:, None], np.stack([v00, v10, v11], 1), np.stack([v01, v10, v11], 1))
    el = np.empty((2 * ci.size, 3), dtype=np.int64)
    el[0::2], el[1::2] = t0, t1
    m = SimplexMesh(2, verts, np.sort(el, axis=1))
    i0 = int(np.argmin(np.abs(xi)))
    j0 = int(np.argmin(np.abs(s - tip)))
    m.info.update(dict(fault_column=i0, fault_tip_row=j0, nx=nx, ns=ns, dip=theta, xi=xi, s=s))

    def boundary_bc(c):
        top = np.all(np.abs(c[:, :, 1]) < 1e-9, axis=1)
        return np.where(top, BC_NATURAL, BC_DIRICHLET)

    def interior_bc(c):
        # vertices on the fault grid line: xi == 0 and s >= tip
        ids_xi = c[:, :, 0] + c[:, :, 1] / np.tan(theta)
        on = np.all(np.abs(ids_xi) < 1e-9, axis=1) & np.all(c[:, :, 1] >= tip - 1e-9, axis=1)
        return np.where(on, BC_FAULT, BC_NONE)

    m.info["boundary_bc"], m.info["interior_bc"] = boundary_bc, interior_bc
    return m


def fault_facets(mesh: SimplexMesh) -> np.ndarray:
    """Fault facet numbers ordered by depth (surface first)."""
    f = np.nonzero(mesh.facet_bc == BC_FAULT)[0]
    depth = mesh.vertices[mesh.facets[f]][:, :, 1].mean(axis=1)
    return f[np.argsort(-depth)]


def topology(mesh: SimplexMesh, boundary_bc: Callable[[np.ndarray], np.ndarray] | int = BC_DIRICHLET,
             interior_bc: Callable[[np.ndarray], np.ndarray] | None = None) -> SimplexMesh:
    """Facets and FacetInfo arrays.  boundary_bc maps facet vertex coordinates [F, D, D] to BC
    codes (or is a constant); interior_bc likewise marks interior facets (e.g. faults)."""
    D = mesh.dim
    nf = D + 1
    E = mesh.num_elements
    fv = facet_vertices(D)
    faces = np.stack([mesh.elements[:, list(v)] for v in fv], axis=1).reshape(E * nf, D)
    uniq, inv = np.unique(faces, axis=0, return_inverse=True)
    inv = inv.ravel()
    F = uniq.shape[0]
    elem_of = np.repeat(np.arange(E, dtype=np.int64), nf)
    local_of = np.tile(np.arange(nf, dtype=np.int32), E)
    order = np.lexsort((elem_of, inv))
    inv_s, el_s, lo_s = inv[order], elem_of[order], local_of[order]
    first = np.ones(inv_s.size, dtype=bool)
    first[1:] = inv_s[1:] != inv_s[:-1]
    counts = np.bincount(inv_s, minlength=F)
    if counts.max() > 2:
        raise ValueError("non-manifold mesh: a facet has more than two elements")
    up = np.empty((F, 2), dtype=np.int64)
    loc = np.empty((F, 2), dtype=np.int32)
    fidx = inv_s[first]
    up[fidx, 0] = el_s[first]
    loc[fidx, 0] = lo_s[first]
    up[:, 1] = up[:, 0]
    loc[:, 1] = loc[:, 0]
    second = ~first
    up[inv_s[second], 1] = el_s[second]
    loc[inv_s[second], 1] = lo_s[second]
    boundary = counts == 1
    bc = np.zeros(F, dtype=np.int32)
    coords = mesh.vertices[uniq]  # [F, D, D]
    if callable(boundary_bc):
        bc[boundary] = np.asarray(boundary_bc(coords[boundary]), dtype=np.int32)
    else:
        bc[boundary] = int(boundary_bc)
    if interior_bc is not None:
        ib = np.asarray(interior_bc(coords[~boundary]), dtype=np.int32)
        bc[~boundary] = ib
    mesh.facets, mesh.facet_up, mesh.facet_local, mesh.facet_bc = uniq, up, loc, bc
    return mesh


def p2_nodes(mesh: SimplexMesh, surface: Callable[[np.ndarray], np.ndarray] | None = None):
    """P2 element nodes (vertices, then edge midpoints in VTK order) interpolating a curved
    boundary: surface(x) returns the displacement of boundary points x [M, D] (zero inside).
    Vertices and the midpoints of edges lying on a boundary plane are moved onto the surface; all
    other edges stay straight between their (moved) end points."""
    D = mesh.dim
    X = mesh.vertices[mesh.elements]  # [E, D+1, D]
    Xd = X if surface is None else X + surface(X.reshape(-1, D)).reshape(X.shape)
    mids = []
    for (i, j) in EDGES[D]:
        a, b = X[:, i], X[:, j]
        m = 0.5 * (Xd[:, i] + Xd[:, j])
        if surface is not None:
            on = _same_boundary_plane(a, b)
            mm = 0.5 * (a[on] + b[on])
            m[on] = mm + surface(mm)
        mids.append(m)
    return np.concatenate([Xd, np.stack(mids, axis=1)], axis=1)


def _same_boundary_plane(a: np.ndarray, b: np.ndarray, tol: float = 1e-12) -> np.ndarray:
    on = np.zeros(a.shape[0], dtype=bool)
    for d in range(a.shape[1]):
        for c in (0.0, 1.0):
            on |= (np.abs(a[:, d] - c) < tol) & (np.abs(b[:, d] - c) < tol)
    return on


def geometry_nodes(mesh: SimplexMesh, degree: int, p2: np.ndarray | None = None,
                   transform: Callable[[np.ndarray], np.ndarray] | None = None, tables=None) -> SimplexMesh:
    """Degree-N warp & blend geometry nodes of every element (Curvilinear::vertices).  tables: an
    object with ref_nodes / ref_basis of this module's signatures (default: the native library's)."""
    D = mesh.dim
    rn, rb = (ref_nodes, ref_basis) if tables is None else (tables.ref_nodes, tables.ref_basis)
    xi = rn(D, degree, WARP_BLEND)  # [Ngeo, D]
    if p2 is None:
        lam = np.concatenate([(1.0 - xi.sum(axis=1))[:, None], xi], axis=1)  # [Ngeo, D+1]
        X = mesh.vertices[mesh.elements]  # [E, D+1, D]
        nodes = np.einsum("nv,evd->end", lam, X)
    else:
        phi = rb(D, 2, EQUIDISTANT, xi)  # [nP2, Ngeo]
        nodes = np.einsum("jn,ejd->end", phi, p2)
        mesh.p2_nodes = p2
    if transform is not None:
        nodes = transform(nodes.reshape(-1, D)).reshape(nodes.shape)
    mesh.geo_degree = degree
    mesh.geo_nodes = np.ascontiguousarray(nodes)
    return mesh


def box_boundary_surface(amplitude: float = 0.02):
    """Smooth displacement of the faces of the unit square / cube: on the face x_d = c a point
    moves by amplitude * prod_k sin(pi x_k) (k over the in-face coordinates) along the outward
    normal.  It vanishes on the box's edges and corners, so neighbouring faces stay conforming."""
    def surface(x: np.ndarray) -> np.ndarray:
        out = np.zeros_like(x)
        D = x.shape[1]
        tol = 1e-12
        for d in range(D):
            o = [k for k in range(D) if k != d]
            bump = amplitude * np.prod(np.sin(np.pi * x[:, o]), axis=1)
            for c, sgn in ((0.0, -1.0), (1.0, 1.0)):
                on = np.abs(x[:, d] - c) < tol
                out[on, d] += sgn * bump[on]
        return out
    return surface


def build(mesh: SimplexMesh, degree: int, boundary_bc=BC_DIRICHLET, interior_bc=None, curve=None,
          transform=None, tables=None) -> SimplexMesh:
    """Topology + geometry nodes in one call; curve is a boundary displacement (P2 geometry)."""
    topology(mesh, boundary_bc, interior_bc)
    p2 = p2_nodes(mesh, curve) if curve is not None else None
    return geometry_nodes(mesh, degree, p2, transform, tables)


def union(meshes: list[SimplexMesh]) -> tuple[SimplexMesh, np.ndarray]:
    """Disjoint union of meshes that already carry topology and geometry nodes: one operator over
    the union is block diagonal with one block per mesh.  Returns the union and the element offsets
    [0, E_0, E_0 + E_1, ...]."""
    D = meshes[0].dim
    eoff = np.cumsum([0] + [m.num_elements for m in meshes]).astype(np.int64)
    voff = np.cumsum([0] + [m.vertices.shape[0] for m in meshes]).astype(np.int64)
    u = SimplexMesh(D, np.concatenate([m.vertices for m in meshes]),
                    np.concatenate([m.elements + voff[i] for i, m in enumerate(meshes)]))
    u.facets = np.concatenate([m.facets + voff[i] for i, m in enumerate(meshes)])
    u.facet_up = np.concatenate([m.facet_up + eoff[i] for i, m in enumerate(meshes)])
    u.facet_local = np.concatenate([m.facet_local for m in meshes])
    u.facet_bc = np.concatenate([m.facet_bc for m in meshes])
    degs = {m.geo_degree for m in meshes}
    if len(degs) != 1:
        raise ValueError("meshes must share the geometry degree")
    u.geo_degree = degs.pop()
    u.geo_nodes = np.concatenate([m.geo_nodes for m in meshes])
    return u, eoff
