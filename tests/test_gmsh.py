"""GMSH (MSH 2.x ASCII) reader: meshes written in GMSH's conventions -- shuffled corner orders,
GMSH's quadratic-tetrahedron edge order, boundary codes as physical tags -- read back into the same
geometry, facet codes and operator (tandem's GMSHParser / GlobalSimplexMeshBuilder behaviour)."""
import numpy as np
import pytest

from cases import tandem_quadrature
from oracle import Oracle
from tandem_b200 import gmsh
from tandem_b200 import mesh as M
from tandem_b200.operator import ELASTICITY


def _facet_table(m, vertices=None):
    """(sorted facet centroids, their codes) -- independent of vertex numbering."""
    c = (m.vertices if vertices is None else vertices)[m.facets].mean(axis=1)
    o = np.lexsort(tuple(np.round(c, 12).T))
    return c[o], m.facet_bc[o]


def test_linear_triangles_with_boundary_codes(tmp_path):
    def bbc(c):
        top = np.all(np.abs(c[:, :, 1] - 1.0) < 1e-12, axis=1)
        return np.where(top, M.BC_NATURAL, M.BC_DIRICHLET)

    ref = M.build(M.square_mesh(4), 2, boundary_bc=bbc)
    perm = np.random.default_rng(0).permuted(np.tile(np.arange(3), (ref.num_elements, 1)), axis=1)
    p = str(tmp_path / "sq.msh")
    gmsh.write_msh(p, ref, corner_perm=perm)
    m = gmsh.read_msh(p, 2, 2)
    assert m.num_elements == ref.num_elements and m.num_facets == ref.num_facets
    c0, b0 = _facet_table(ref)
    c1, b1 = _facet_table(m)
    np.testing.assert_allclose(c1, c0, atol=1e-14)
    np.testing.assert_array_equal(b1, b0)
    assert m.info["unknown_bc"] == 0
    for e in range(m.num_elements):  # same node sets per element
        a = np.round(np.sort(ref.geo_nodes[e], axis=0), 12)
        b = np.round(np.sort(m.geo_nodes[e], axis=0), 12)
        np.testing.assert_allclose(np.sort(b.view([("", float)] * 2), axis=0).view(float),
                                   np.sort(a.view([("", float)] * 2), axis=0).view(float), atol=1e-12)


def _invariants(m, degree):
    """u^T A u and u^T b for u the nodal interpolant of a smooth field (independent of numbering)."""
    q = tandem_quadrature(3, degree)
    orc = Oracle(m, degree, ELASTICITY, q)
    X = orc.volume_coords()
    orc.set_material(2.0 + X[..., 0], 1.0 + 0.5 * X[..., 1])
    nodes = m.geo_nodes  # degree-N warp & blend nodes = the nodal DOF positions (geo degree N)
    f = np.stack([np.sin(nodes[..., 0] + 0.3 * nodes[..., 1]), np.cos(nodes[..., 2]), nodes[..., 0] * nodes[..., 1]],
                 axis=1)  # [E, Q, Nbf]
    u = np.ascontiguousarray(f).reshape(-1)
    Xf = orc.facet_coords()
    g = np.ascontiguousarray(np.stack([np.cos(Xf[..., 0]), Xf[..., 1], 0 * Xf[..., 2]], axis=1))
    b = orc.rhs(None, g)
    return u @ orc.apply(u), u @ b


def test_quadratic_tetrahedra_reproduce_the_curved_geometry_and_operator(tmp_path):
    deg = 3
    ref = M.build(M.cube_mesh(2), deg, curve=M.box_boundary_surface(0.02))
    perm = np.random.default_rng(1).permuted(np.tile(np.arange(4), (ref.num_elements, 1)), axis=1)
    p = str(tmp_path / "cube.msh")
    gmsh.write_msh(p, ref, p2=ref.p2_nodes, corner_perm=perm)
    m = gmsh.read_msh(p, 3, deg)
    moved = ref.vertices + M.box_boundary_surface(0.02)(ref.vertices)
    c0, b0 = _facet_table(ref, moved)
    c1, b1 = _facet_table(m)
    np.testing.assert_allclose(c1, c0, atol=1e-14)
    np.testing.assert_array_equal(b1, b0)
    for e in range(m.num_elements):
        a = ref.geo_nodes[e][np.lexsort(tuple(np.round(ref.geo_nodes[e], 10).T))]
        b = m.geo_nodes[e][np.lexsort(tuple(np.round(m.geo_nodes[e], 10).T))]
        np.testing.assert_allclose(b, a, atol=1e-13)
    q0, r0 = _invariants(ref, deg)
    q1, r1 = _invariants(m, deg)
    assert abs(q1 - q0) <= 1e-12 * abs(q0) and abs(r1 - r0) <= 1e-12 * abs(r0)


def test_rejected_and_ignored_input(tmp_path):
    ref = M.build(M.square_mesh(2), 1)
    p = str(tmp_path / "a.msh")
    gmsh.write_msh(p, ref)
    text = open(p).read()
    with pytest.raises(ValueError, match="unsupported MSH version"):
        gmsh.read_msh(text.replace("2.2 0 8", "4.1 0 8"), 2, 1, from_text=True)
    lines = text.splitlines()
    i = lines.index("$Elements")
    first = lines[i + 2].split()
    mixed = " ".join([first[0], "9", "2", "1", "1"] + first[5:] + ["1", "2", "3"])
    with pytest.raises(ValueError, match="mixed meshes"):
        gmsh.read_msh("\n".join(lines[:i + 2] + [mixed] + lines[i + 3:]), 2, 1, from_text=True)
    # an unknown physical tag on a facet counts and leaves the facet at None
    j = next(k for k in range(i + 2, len(lines)) if lines[k].split()[1] == "1")
    w = lines[j].split()
    w[3] = w[4] = "7"
    m = gmsh.read_msh("\n".join(lines[:j] + [" ".join(w)] + lines[j + 1:]), 2, 1, from_text=True)
    assert m.info["unknown_bc"] == 1 and np.sum(m.facet_bc == M.BC_NONE) == np.sum(ref.facet_bc == M.BC_NONE) + 1


EXAMPLE = "/root/reference/examples/poisson/2d/embedded_half.msh"


@pytest.mark.skipif(not __import__("os").path.exists(EXAMPLE), reason="reference example mesh not present")
def test_reference_example_mesh_reads_into_an_operator():
    """tandem's own example mesh (examples/poisson/2d/embedded_half.msh, MSH 2.2 with physical
    tags 1 / 3 / 5 on its lines): read, then the oracle's operator on it is symmetric and positive
    on random vectors."""
    m = gmsh.read_msh(EXAMPLE, 2, 2)
    assert m.num_elements == 23 and m.info["unknown_bc"] == 0
    codes, counts = np.unique(m.facet_bc, return_counts=True)
    assert dict(zip(codes.tolist(), counts.tolist())) == {0: 29, 1: 4, 3: 1, 5: 5}
    q = tandem_quadrature(2, 2)
    from tandem_b200.operator import POISSON
    orc = Oracle(m, 2, POISSON, q)
    orc.set_material(np.ones(orc.volume_coords().shape[:2]))
    rng = np.random.default_rng(3)
    x, z = rng.standard_normal(orc.ndof), rng.standard_normal(orc.ndof)
    assert abs(z @ orc.apply(x) - x @ orc.apply(z)) <= 1e-12 * np.linalg.norm(z) * np.linalg.norm(orc.apply(x))
    assert x @ orc.apply(x) > 0
