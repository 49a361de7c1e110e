"""Host side of the p-multigrid preconditioner: level degrees (tandem's MGConfig::levels) and the
reference interpolation matrices (NodalInterpolation / ModalInterpolation) against the oracle's
restatement, and the interpolation's defining property (exact embedding of the coarse space)."""
import numpy as np
import pytest

import oracle
from tandem_b200.operator import ELASTICITY, POISSON, mg_interpolation, mg_level_degrees
from tandem_b200.refelem import ref_nodes


@pytest.mark.parametrize("strategy", ["twolevel", "logarithmic", "full"])
def test_level_degrees_match_mgconfig(strategy):
    code = ("twolevel", "logarithmic", "full").index(strategy)
    for coarse in (0, 1, 2):
        for N in range(1, 9):
            assert mg_level_degrees(strategy, coarse, N) == oracle.mg_levels(code, coarse, N)


def test_level_degrees_known_values():
    # MGConfig::levels by hand: logarithmic halves the degree, a coarse level >= N becomes N - 1
    assert mg_level_degrees("logarithmic", 1, 4) == [1, 2, 4]
    assert mg_level_degrees("logarithmic", 1, 5) == [1, 2, 5]
    assert mg_level_degrees("logarithmic", 1, 8) == [1, 2, 4, 8]
    assert mg_level_degrees("logarithmic", 1, 1) == [0, 1]
    assert mg_level_degrees("full", 1, 4) == [1, 2, 3, 4]
    assert mg_level_degrees("twolevel", 1, 4) == [1, 4]
    assert mg_level_degrees("twolevel", 3, 2) == [1, 2]


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("kind", [POISSON, ELASTICITY])
def test_interpolation_matches_oracle(dim, kind):
    for n_to in range(1, 5):
        for n_from in range(n_to):
            a = mg_interpolation(dim, kind, n_to, n_from)
            b = oracle.mg_interpolation(dim, kind, n_to, n_from)
            assert a.shape == b.shape
            assert np.abs(a - b).max() < 1e-13, (n_to, n_from)


@pytest.mark.parametrize("dim", [2, 3])
def test_nodal_interpolation_embeds_the_coarse_space(dim):
    """Coarse nodal values of a degree-n_from polynomial, interpolated, equal the polynomial at the
    fine nodes (the rows are the coarse Lagrange basis at the fine nodes)."""
    rng = np.random.default_rng(dim)
    for n_to in range(2, 5):
        for n_from in range(1, n_to):
            c = rng.standard_normal(4)

            def poly(X):
                s = sum(X[:, i] for i in range(dim))
                return c[0] + c[1] * X[:, 0] + c[2] * s ** n_from + c[3] * X[:, 1] ** max(n_from - 1, 0)

            I = mg_interpolation(dim, ELASTICITY, n_to, n_from)
            got = I @ poly(ref_nodes(dim, n_from))
            assert np.abs(got - poly(ref_nodes(dim, n_to))).max() < 1e-12


def test_modal_interpolation_is_injection():
    I = mg_interpolation(3, POISSON, 4, 2)
    assert np.array_equal(I[:10], np.eye(10)) and not I[10:].any()


def _op(m, dim, degree=2):
    from cases import tandem_quadrature
    from tandem_b200.operator import DGOperator
    return DGOperator(m, degree, ELASTICITY, tandem_quadrature(dim, degree))


def _closed_neighbourhoods(m):
    E = m.num_elements
    nb = [{e} for e in range(E)]
    for a, b in m.facet_up:
        if a != b:
            nb[a].add(int(b))
            nb[b].add(int(a))
    return nb


@pytest.mark.parametrize("dim,n", [(2, 5), (3, 3)])
def test_probing_colouring_is_distance_two(dim, n):
    """Every closed neighbourhood (an element and the elements across its interior facets) holds
    each colour at most once, which is what lets one probe recover every block of a colour."""
    from tandem_b200 import mesh as M
    m = M.build(M.square_mesh(n) if dim == 2 else M.cube_mesh(n), 2)
    col, nc = _op(m, dim).mg_colouring()
    assert col.min() == 0 and col.max() == nc - 1
    for hood in _closed_neighbourhoods(m):
        cs = [col[e] for e in hood]
        assert len(set(cs)) == len(cs)


def test_vertex_numbering_follows_facet_connectivity():
    """Connected mesh: the numbering is the mesh's own vertex ids up to renaming.  Mesh union of
    overlapping copies: no vertex is shared between problems (they stay independent)."""
    from tandem_b200 import mesh as M
    m = M.build(M.square_mesh(4), 2)
    vid, nv = _op(m, 2).mg_vertex_numbering()
    pairs = set(zip(m.elements.ravel().tolist(), vid.ravel().tolist()))
    assert nv == len(np.unique(m.elements)) == len(pairs)
    meshes = [M.build(M.square_mesh(k), 2) for k in (3, 2, 3)]
    um, eoff = M.union(meshes)
    vid, nv = _op(um, 2).mg_vertex_numbering()
    seen = []
    for i in range(len(meshes)):
        part = vid[eoff[i]:eoff[i + 1]]
        assert len(np.unique(part)) == len(np.unique(meshes[i].elements))
        seen.append(set(part.ravel().tolist()))
    assert sum(len(s) for s in seen) == nv == len(set().union(*seen))


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("kind", [POISSON, ELASTICITY])
def test_p1_embedding_reproduces_hat_functions(dim, kind):
    """Evaluated at random points, the degree-p function with the embedding's coefficients equals
    the corner's barycentric coordinate (exact for every p >= 1)."""
    from tandem_b200.operator import mg_p1_embedding
    from tandem_b200.refelem import MODAL, WARP_BLEND, ref_basis
    rng = np.random.default_rng(dim + 10 * kind)
    pts = rng.dirichlet(np.ones(dim + 1), size=20)[:, 1:]
    lam = np.concatenate([1.0 - pts.sum(axis=1, keepdims=True), pts], axis=1)  # [np, dim + 1]
    for p in range(1, 5):
        T = mg_p1_embedding(dim, kind, p)
        Eb = ref_basis(dim, p, MODAL if kind == POISSON else WARP_BLEND, pts)  # [Nbf, np]
        assert np.abs(Eb.T @ T - lam).max() < 1e-12, p
