"""GMSH mesh files (MSH 2.x ASCII) for the operator: tandem's GMSHParser + GlobalSimplexMeshBuilder
(src/io/GMSHParser.cpp, src/io/GlobalSimplexMeshBuilder.cpp) restated for this package.

* $Nodes: node tags 1..n with x y z; $Elements: tag, type, number of tags, tags, nodes.
* Elements of the domain dimension (triangles in 2D, tetrahedra in 3D) are the mesh, linear
  (types 2 / 4) or quadratic (types 9 / 11; their edge nodes become the P2 geometry); mixing
  orders is an error, as in tandem.  The first tag is the element's volume tag.
* Elements of one dimension less carry the facet's boundary condition in their first (physical)
  tag, with tandem's codes (0 None, 1 Natural, 3 Fault, 5 Dirichlet); other codes count as
  unknown and leave the facet at None.  Facets of the mesh that the file does not list are None.
* Lower-dimensional elements (points, and lines in 3D) are ignored.
* Vertices are renumbered in order of first appearance among the elements' corners, quadratic
  edge nodes are dropped from the vertex list (they only shape the geometry), and each element's
  corners are sorted by vertex id with its edge nodes permuted along (tandem permutes its
  high-order nodes to the sorted vertex order the same way).
"""
from __future__ import annotations

import numpy as np

from . import mesh as M

# element types: (dimension, corners, total nodes)
_TYPES = {1: (1, 2, 2), 8: (1, 2, 3), 2: (2, 3, 3), 9: (2, 3, 6), 4: (3, 4, 4), 11: (3, 4, 10), 15: (0, 1, 1)}
# edge order of GMSH's quadratic simplices (gmsh.info, "Node ordering"); tandem's
# NumberingConvention.h lists the same tetrahedron edges
_GMSH_EDGES = {2: [(0, 1), (1, 2), (2, 0)], 3: [(0, 1), (1, 2), (2, 0), (3, 0), (3, 2), (3, 1)]}
_BC_CODES = (M.BC_NONE, M.BC_NATURAL, M.BC_FAULT, M.BC_DIRICHLET)


def parse_msh(text: str, dim: int) -> dict:
    """Parses MSH 2.x ASCII; returns nodes [n, 3], domain elements (type, tags, nodes) and facet
    elements (tags, corner nodes), all node ids 0-based."""
    tok = text.split()
    pos = 0

    def expect(word):
        nonlocal pos
        if pos >= len(tok) or tok[pos] != word:
            raise ValueError(f"expected {word} at token {pos}")
        pos += 1

    expect("$MeshFormat")
    version = float(tok[pos])
    if not (2.0 <= version < 3.0):
        raise ValueError(f"unsupported MSH version {version:.1f} (2.x ASCII is read)")
    if tok[pos + 1] != "0":
        raise ValueError("binary MSH files are not supported")
    pos += 3
    expect("$EndMeshFormat")
    nodes = None
    vol_type, vol_tags, vol_nodes, fct_tags, fct_nodes = None, [], [], [], []
    while pos < len(tok):
        if tok[pos] == "$Nodes":
            pos += 1
            n = int(tok[pos])
            pos += 1
            rec = np.array(tok[pos:pos + 4 * n], dtype=np.float64).reshape(n, 4)
            pos += 4 * n
            ids = rec[:, 0].astype(np.int64)
            if ids.min() < 1 or ids.max() > n:
                raise ValueError(f"node tags must lie in 1..{n}")
            nodes = np.zeros((n, 3))
            nodes[ids - 1] = rec[:, 1:]
            expect("$EndNodes")
        elif tok[pos] == "$Elements":
            pos += 1
            n = int(tok[pos])
            pos += 1
            for _ in range(n):
                etype = int(tok[pos + 1])
                ntags = int(tok[pos + 2])
                tags = [int(t) for t in tok[pos + 3:pos + 3 + ntags]]
                pos += 3 + ntags
                if etype not in _TYPES:
                    raise ValueError(f"GMSH element type {etype} is not a linear or quadratic simplex")
                edim, _, nn = _TYPES[etype]
                enodes = [int(t) - 1 for t in tok[pos:pos + nn]]
                pos += nn
                tag = tags[0] if tags else -1
                if edim == dim:
                    if vol_type is None:
                        vol_type = etype
                    elif vol_type != etype:
                        raise ValueError(f"element of type {etype} conflicts with previous type {vol_type} "
                                         "(mixed meshes are not supported)")
                    vol_tags.append(tag)
                    vol_nodes.append(enodes)
                elif edim == dim - 1:
                    fct_tags.append(tag)
                    fct_nodes.append(enodes[:dim])
                elif edim > dim:
                    raise ValueError(f"element of type {etype} has dimension {edim} > {dim}")
            expect("$EndElements")
        else:
            pos += 1
    if nodes is None or vol_type is None:
        raise ValueError(f"the file has no nodes or no {dim}-simplices")
    return dict(nodes=nodes, vol_type=vol_type, vol_tags=np.array(vol_tags, dtype=np.int64),
                vol_nodes=np.array(vol_nodes, dtype=np.int64), fct_tags=np.array(fct_tags, dtype=np.int64),
                fct_nodes=np.array(fct_nodes, dtype=np.int64).reshape(-1, dim))


def read_msh(source: str, dim: int, degree: int, from_text: bool = False) -> M.SimplexMesh:
    """Mesh (topology, boundary conditions, geometry nodes of the given polynomial degree) from a
    MSH 2.x file (or its text)."""
    text = source if from_text else open(source).read()
    p = parse_msh(text, dim)
    vn = p["vol_nodes"]
    corners = vn[:, :dim + 1]
    # vertices in order of first appearance among the corners
    flat = corners.ravel()
    uniq, first = np.unique(flat, return_index=True)
    order = uniq[np.argsort(first)]
    new_id = np.full(p["nodes"].shape[0], -1, dtype=np.int64)
    new_id[order] = np.arange(order.size)
    vertices = np.ascontiguousarray(p["nodes"][order, :dim])
    C = new_id[corners]
    perm = np.argsort(C, axis=1, kind="stable")
    S = np.take_along_axis(C, perm, axis=1)
    mesh = M.SimplexMesh(dim, vertices, S)
    # boundary conditions from the facet elements
    fc = new_id[p["fct_nodes"]]
    known = np.all(fc >= 0, axis=1)
    fc = np.sort(fc[known], axis=1)
    tags = p["fct_tags"][known]
    bc = np.where(np.isin(tags, _BC_CODES), tags, M.BC_NONE).astype(np.int32)
    M.topology(mesh, boundary_bc=M.BC_NONE)
    V = vertices.shape[0]
    key = lambda a: np.ravel_multi_index(tuple(a.T), (V,) * dim)  # noqa: E731
    fkey = key(mesh.facets)
    lookup = dict(zip(key(fc).tolist(), bc.tolist())) if len(fc) else {}
    mesh.facet_bc = np.array([lookup.get(k, M.BC_NONE) for k in fkey.tolist()], dtype=np.int32)
    mesh.info.update(volume_tags=p["vol_tags"], unknown_bc=int(np.sum(~np.isin(tags, _BC_CODES))),
                     source_type=int(p["vol_type"]))
    # quadratic geometry: edge nodes in this package's P2 order for the sorted corners
    p2 = None
    if vn.shape[1] > dim + 1:
        X = p["nodes"][:, :dim]
        N = p["nodes"].shape[0]
        ge = _GMSH_EDGES[dim]
        ekey = np.stack([np.minimum(corners[:, a], corners[:, b]) * N + np.maximum(corners[:, a], corners[:, b])
                         for a, b in ge], axis=1)
        sorted_orig = np.take_along_axis(corners, perm, axis=1)
        mids = []
        for i, j in M.EDGES[dim]:
            a, b = sorted_orig[:, i], sorted_orig[:, j]
            want = np.minimum(a, b) * N + np.maximum(a, b)
            k = np.argmax(ekey == want[:, None], axis=1)
            if not np.all(ekey[np.arange(len(k)), k] == want):
                raise ValueError("inconsistent quadratic element")
            mids.append(X[vn[np.arange(len(k)), dim + 1 + k]])
        p2 = np.concatenate([vertices[S], np.stack(mids, axis=1)], axis=1)
    return M.geometry_nodes(mesh, degree, p2)


def write_msh(path: str, mesh: M.SimplexMesh, p2: np.ndarray | None = None, facet_tags=None,
              corner_perm: np.ndarray | None = None) -> None:
    """Writes the mesh (and its facets whose code is not None, or `facet_tags` for all facets) as
    MSH 2.2 ASCII; with p2 [E, nP2, D] (vertices then edges in this package's order) quadratic
    elements in GMSH's edge order.  corner_perm [E, D+1] lists each element's corners in another
    order (the file then differs from the mesh only in that order)."""
    D = mesh.dim
    V = mesh.vertices.shape[0]
    verts = mesh.vertices.copy()
    if p2 is not None:  # the curved geometry may move vertices too
        verts[mesh.elements.ravel()] = p2[:, :D + 1].reshape(-1, D)
    nodes = [np.pad(verts, ((0, 0), (0, 3 - D)))]
    elems = []
    if p2 is not None:
        E = mesh.num_elements
        ne = len(M.EDGES[D])
        mid = np.pad(p2[:, D + 1:].reshape(-1, D), ((0, 0), (0, 3 - D)))
        nodes.append(mid)
        mid_id = V + np.arange(E * ne).reshape(E, ne)
        pos = {e: k for k, e in enumerate(M.EDGES[D])}
        for e in range(E):
            c = mesh.elements[e]
            pe = range(D + 1) if corner_perm is None else corner_perm[e]
            loc = [int(a) for a in pe]
            ids = [int(c[a]) for a in loc]
            for a, b in _GMSH_EDGES[D]:
                i, j = loc[a], loc[b]
                k = pos.get((i, j), pos.get((j, i)))
                ids.append(int(mid_id[e, k]))
            elems.append((9 if D == 2 else 11, 1, ids))
    else:
        for e, c in enumerate(mesh.elements):
            pe = range(D + 1) if corner_perm is None else corner_perm[e]
            elems.append((2 if D == 2 else 4, 1, [int(c[a]) for a in pe]))
    tags = mesh.facet_bc if facet_tags is None else np.asarray(facet_tags)
    for f in range(mesh.num_facets):
        if facet_tags is None and tags[f] == M.BC_NONE:
            continue
        elems.append((1 if D == 2 else 2, int(tags[f]), [int(v) for v in mesh.facets[f]]))
    X = np.concatenate(nodes)
    with open(path, "w") as fh:
        fh.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(X))
        for i, x in enumerate(X):
            fh.write("%d %.17g %.17g %.17g\n" % (i + 1, x[0], x[1], x[2]))
        fh.write("$EndNodes\n$Elements\n%d\n" % len(elems))
        for i, (t, tag, ids) in enumerate(elems):
            fh.write("%d %d 2 %d %d %s\n" % (i + 1, t, tag, tag, " ".join(str(v + 1) for v in ids)))
        fh.write("$EndElements\n")
