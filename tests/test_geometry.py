"""Curvilinear geometry of the host set-up: tandem's known answers (test/geometry.cpp:27-110) and
agreement with the oracle's independent restatement."""
import numpy as np
import pytest

from cases import make_mesh, product_and_oracle, tandem_quadrature
from tandem_b200 import mesh as M
from tandem_b200.operator import DGOperator, Quadrature, POISSON, ELASTICITY

C45, S45 = np.cos(3.14159265359 / 4.0), np.sin(3.14159265359 / 4.0)


def _rotated_unit_mesh():
    m = M.square_mesh(1)

    def transform(v):
        x, y = 2.0 * v[:, 0] - 1.0, 2.0 * v[:, 1] - 1.0
        return np.stack([C45 * x - S45 * y, C45 * x + S45 * y], axis=1)

    M.topology(m, M.BC_DIRICHLET)
    return M.geometry_nodes(m, 1, transform=transform)


def test_curvilinear_map_kat():
    m = _rotated_unit_mesh()
    quad = Quadrature(np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]), np.ones(3) / 6, np.array([[0.0]]), np.ones(1))
    op = DGOperator(m, 1, POISSON, quad)
    X = op.volume_coords()
    expect = {0: [(-1, -1), (1, -1), (-1, 1)], 1: [(1, -1), (-1, 1), (1, 1)]}
    for el, pts in expect.items():
        for q, (a, b) in enumerate(pts):
            np.testing.assert_allclose(X[el, q], [C45 * a - S45 * b, C45 * a + S45 * b], atol=1e-12)


def test_curvilinear_normals_kat():
    m = _rotated_unit_mesh()
    quad = Quadrature(np.array([[1 / 3, 1 / 3]]), np.array([0.5]), np.array([[0.0]]), np.ones(1))
    op = DGOperator(m, 1, POISSON, quad)
    n = op.facet_normals()[:, 0, :]
    r2 = np.sqrt(2.0)
    # (element, local face) -> expected side-0 normal at chi = 0 (test/geometry.cpp:79-90)
    expect = {(0, 0): (r2, -r2), (0, 1): (-r2, -r2), (0, 2): (0.0, 2 * r2),
              (1, 1): (r2, r2), (1, 2): (-r2, r2)}
    for f in range(m.num_facets):
        key = (int(m.facet_up[f, 0]), int(m.facet_local[f, 0]))
        np.testing.assert_allclose(n[f], expect[key], atol=1e-9)


@pytest.mark.parametrize("kind,dim,curved", [(POISSON, 2, False), (ELASTICITY, 2, True), (ELASTICITY, 3, True),
                                              (POISSON, 3, True)])
def test_host_setup_matches_oracle(kind, dim, curved):
    m, op, orc = product_and_oracle(kind, dim, 3 if dim == 2 else 2, 4, curved, True)
    np.testing.assert_allclose(op.volume_coords(), orc.volume_coords(), atol=1e-14)
    np.testing.assert_allclose(op.facet_coords(), orc.facet_coords(), atol=1e-14)
    np.testing.assert_allclose(op.facet_normals(), orc.facet_normals(), rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(op.penalty(), orc.penalty(), rtol=1e-11)
    np.testing.assert_allclose(op.material_nodal(0), orc.material_nodal(0), rtol=1e-11, atol=1e-12)
    if kind == ELASTICITY:
        np.testing.assert_allclose(op.material_nodal(1), orc.material_nodal(1), rtol=1e-11, atol=1e-12)


def test_curved_geometry_is_conforming():
    """Shared P2 edges get identical midpoints from every element that holds them."""
    m = make_mesh(3, 3, 4, curved=True)
    p2 = m.p2_nodes
    edges = M.EDGES[3]
    seen = {}
    for e in range(m.num_elements):
        for k, (i, j) in enumerate(edges):
            key = tuple(sorted((int(m.elements[e, i]), int(m.elements[e, j]))))
            mid = p2[e, 4 + k]
            if key in seen:
                np.testing.assert_allclose(mid, seen[key], atol=1e-15)
            else:
                seen[key] = mid


def test_volume_of_curved_cube():
    """Sum of element volumes = 1 + the bulge of the six curved faces (2 * amplitude * (2/pi)^2 each
    side pair, integrated over the P2 interpolant only approximately)."""
    m = make_mesh(3, 4, 4, curved=True)
    q = tandem_quadrature(3, 4)
    op = DGOperator(m, 4, POISSON, q)
    from oracle import Oracle
    orc = Oracle(m, 4, POISSON, q)
    X = orc.volume_coords()
    # integrate 1 with the oracle's error functional: || 0 - 1 ||_L2^2 = volume
    vol = orc.error_L2(np.zeros(orc.ndof), np.ones((orc.E, orc.Nq, 1))) ** 2
    bulge = 6 * 0.02 * (2 / np.pi) ** 2
    assert abs(vol - (1 + bulge)) < 2e-3
    assert X.shape == (m.num_elements, len(q.vol_w), 3)
