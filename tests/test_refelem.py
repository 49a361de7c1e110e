"""Reference-element tables pinned against tandem: its own sources compiled in place
(tests/golden/quadrature.json, dubiner.json) and the known answers of its unit tests
(tests/golden/kat.json from test/basis.cpp, test/quadrules.cpp, test/form.cpp)."""
import numpy as np
import pytest

from cases import golden
from tandem_b200.refelem import EQUIDISTANT, MODAL, WARP_BLEND, conical_rule, ref_basis, ref_nodes


def tandem_order(dim, N):
    """AllIntegerSums<dim>(N) enumeration (src/util/Combinatorics.h:47-115), restated here
    independently of the library to pin its basis ordering."""
    m = [0] * dim
    out = []
    while m[-1] <= N:
        j = [0] * dim
        j[dim - 1] = m[0]
        for k in range(1, dim):
            j[dim - 1 - k] = m[k] - m[k - 1]
        out.append(tuple(j))
        d = 0
        while d < dim - 1 and m[d] == m[d + 1]:
            d += 1
        m[d] += 1
        for k in range(d):
            m[k] = 0
    return out


@pytest.mark.parametrize("dim,key", [(2, "tri"), (3, "tet")])
def test_dubiner_matches_tandem(dim, key):
    order = tandem_order(dim, 4)
    index = {j: i for i, j in enumerate(order)}
    rows = golden("dubiner.json")[key]
    pts = np.array([r["x"] for r in rows])
    E, G = ref_basis(dim, 4, MODAL, pts, grad=True)
    for q, r in enumerate(rows):
        k = index[tuple(r["j"])]
        assert E[k, q] == pytest.approx(r["v"], rel=1e-13, abs=1e-13)
        np.testing.assert_allclose(G[k, :, q], r["g"], rtol=1e-12, atol=1e-12)


def test_basis_order_is_graded():
    assert tandem_order(2, 2) == [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2)]
    assert len(tandem_order(3, 4)) == 35


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("N", [0, 1, 2, 3, 4])
def test_warp_blend_nodes_kat(dim, N):
    ref = np.array(golden("kat.json")["warp_blend"][f"{dim}:{N}"])
    np.testing.assert_allclose(ref_nodes(dim, N, WARP_BLEND), ref, atol=1e-14)


@pytest.mark.parametrize("key", ["2:1", "2:2", "2:3", "2:6", "3:1", "3:2", "3:3", "3:6"])
def test_equidistant_nodes_kat(key):
    dim, N = map(int, key.split(":"))
    ref = np.array(golden("kat.json")["equidistant"][key])
    np.testing.assert_allclose(ref_nodes(dim, N, EQUIDISTANT), ref, atol=1e-14)


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("order", [1, 3, 5, 7, 9, 11])
def test_conical_rule_matches_tandem(dim, order):
    r = golden("quadrature.json")["conical"][f"{dim}:{order}"]
    x, w = conical_rule(dim, order)
    np.testing.assert_allclose(x, np.array(r["points"]).reshape(-1, dim), atol=1e-15)
    np.testing.assert_allclose(w, r["weights"], rtol=1e-13)


def test_conical_triangle_vs_maple():
    k = golden("kat.json")["conical_tri_order3"]
    x, w = conical_rule(2, 3)
    np.testing.assert_allclose(x[:, 0], k["x0"], rtol=1e-12)
    np.testing.assert_allclose(x[:, 1], k["x1"], rtol=1e-12)
    np.testing.assert_allclose(w, k["w"], rtol=1e-12)


def _monomial_exact(x, w, order):
    """tandem's quadrature order test (test/quadrules.cpp:52-83)."""
    from math import factorial, prod
    dim = x.shape[1]
    for j in tandem_order(dim, order):
        val = np.sum(w * np.prod(x ** np.array(j), axis=1))
        js = sorted(j)
        ref = 1.0 / prod(range(js[-1] + 1, sum(js) + dim + 1))
        for d in range(dim - 1):
            ref *= factorial(js[d])
        assert val == pytest.approx(ref, rel=1e-12, abs=1e-15)


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("order", [3, 5, 9])
def test_rules_integrate_monomials(dim, order):
    r = golden("quadrature.json")["auto"][f"{dim}:{order}"]
    _monomial_exact(np.array(r["points"]).reshape(-1, dim), np.array(r["weights"]), order)
    x, w = conical_rule(dim, order)
    _monomial_exact(x, w, order)


def test_autorule_sizes():
    rules = golden("quadrature.json")["auto"]
    for dim, order, size in golden("kat.json")["autorule_sizes"]:
        if f"{dim}:{order}" in rules:
            assert len(rules[f"{dim}:{order}"]["weights"]) == size
    assert len(rules["2:9"]["weights"]) == 19
    assert len(rules["3:9"]["weights"]) == 57
    assert len(rules["1:9"]["weights"]) == 5


def test_modal_mass_matrix_tet_kat():
    """Diagonal modal mass matrix of the unnormalised Dubiner basis (test/form.cpp:19-58)."""
    ref = golden("kat.json")["modal_mass_tet"]
    x, w = conical_rule(3, 6)
    E = ref_basis(3, 3, MODAL, x)
    M = (E * w) @ E.T
    np.testing.assert_allclose(np.diag(M), ref, rtol=1e-12)
    assert np.abs(M - np.diag(np.diag(M))).max() < 1e-14


def test_nodal_basis_is_lagrange():
    for dim in (2, 3):
        nodes = ref_nodes(dim, 4, WARP_BLEND)
        E = ref_basis(dim, 4, WARP_BLEND, nodes)
        np.testing.assert_allclose(E, np.eye(len(nodes)), atol=1e-12)
