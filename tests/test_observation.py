"""Point observation operator of the adjoint study (CPU): P applied to the nodal interpolant of a
linear displacement field reproduces the field at the points (the nodal basis reproduces
polynomials up to its degree), and points outside the mesh are rejected."""
import numpy as np
import pytest
import torch

from tandem_b200 import mesh as M
from tandem_b200 import refelem
from tandem_b200.adjoint import PointObservation


@pytest.mark.parametrize("dim,n,degree", [(2, 4, 3), (3, 3, 4)])
def test_observation_reproduces_linear_fields(dim, n, degree):
    m = M.square_mesh(n) if dim == 2 else M.cube_mesh(n)
    rng = np.random.default_rng(dim)
    pts = rng.uniform(0.1, 0.9, size=(40, dim))
    P = PointObservation(m, degree, pts, device="cpu")
    A = rng.standard_normal((dim, dim))
    c = rng.standard_normal(dim)
    nodes = refelem.ref_nodes(dim, degree)                      # [Nbf][dim]
    V, El = m.vertices, m.elements
    v0 = V[El[:, 0]]
    T = np.transpose(V[El[:, 1:]] - v0[:, None, :], (0, 2, 1))
    X = v0[:, None, :] + np.einsum("eij,kj->eki", T, nodes)     # [E][Nbf][dim]
    F = X @ A.T + c                                             # [E][Nbf][Q]
    u = torch.as_tensor(np.ascontiguousarray(np.transpose(F, (0, 2, 1))).reshape(-1))
    got = P.apply(u).numpy()
    np.testing.assert_allclose(got, pts @ A.T + c, rtol=0, atol=1e-12)


def test_observation_rejects_outside_points():
    m = M.square_mesh(2)
    with pytest.raises(ValueError, match="outside"):
        PointObservation(m, 2, np.array([[1.5, 0.5]]), device="cpu")
