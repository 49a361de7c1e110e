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
