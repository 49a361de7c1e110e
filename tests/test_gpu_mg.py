"""p-multigrid preconditioner on the device against the oracle.

* Galerkin coarse operators (probing of the matrix-free operator, block triple products) equal
  P^T A P of the oracle's dense operator to 1e-12 relative (max norm).
* The Lanczos estimates of lambda_max(D^-1 A_l) lie in [0.7, 1 + 1e-9] x the exact value.
* One V-cycle equals the dense restatement of PCMG's V-cycle (oracle.DenseMultigrid, exact
  coarse solve; the device's coarse CG runs to 1e-13) to 1e-9 relative, with the coarse solve on
  the coarsest DG level or on the continuous P1 level below it.
* Multigrid-preconditioned (flexible) CG solves reach the 1e-10 residual target, checked with the
  oracle's operator, in far fewer iterations than block Jacobi: single problems (FP64 and mixed),
  a segmented batch and multiple right-hand sides."""
import numpy as np
import pytest
import torch

import oracle
from cases import make_mesh, material, mms_inputs, product_and_oracle, tandem_quadrature
from oracle import DenseMultigrid, Oracle, element_interpolation
from tandem_b200 import _ffi
from tandem_b200 import mesh as M
from tandem_b200.operator import DGOperator, ELASTICITY, FP32, FP64, MIXED, POISSON, solve_segmented

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def dev(x):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=DEV)


def dense(orc, n):
    A = np.empty((n, n))
    e = np.zeros(n)
    for j in range(n):
        e[j] = 1.0
        A[:, j] = orc.apply(e)
        e[j] = 0.0
    return A


def prolongations(op, kind, dim, degrees):
    return [element_interpolation(op.E, op.Q, oracle.mg_interpolation(dim, kind, degrees[l + 1], degrees[l]))
            for l in range(len(degrees) - 1)]


def p1_embedding(m, op, kind, dim, degree0):
    """Dense R: continuous P1 (mesh vertices, Q components) -> the coarsest DG level; on element e
    corner i of the (sorted) element, coefficient k of component p gets T[k, i], T the DG basis
    coefficients of the corner's hat function (inverse basis Vandermonde at the warp & blend
    nodes times the barycentric coordinates of those nodes)."""
    from tandem_b200.refelem import MODAL, WARP_BLEND, ref_basis, ref_nodes
    nodes = ref_nodes(dim, degree0)
    Eb = ref_basis(dim, degree0, MODAL if kind == POISSON else WARP_BLEND, nodes)
    Eb = Eb[0] if isinstance(Eb, tuple) else Eb
    lam = np.concatenate([1.0 - nodes.sum(axis=1, keepdims=True), nodes], axis=1)
    T = np.linalg.solve(Eb.T, lam)
    nbf, Q = T.shape[0], op.Q
    nv = int(m.elements.max()) + 1
    R = np.zeros((op.E * nbf * Q, nv * Q))
    for e in range(op.E):
        for i, v in enumerate(m.elements[e]):
            for p in range(Q):
                R[e * nbf * Q + p * nbf:e * nbf * Q + (p + 1) * nbf, v * Q + p] += T[:, i]
    return R


def level_dense(op, level):
    blocks, nbr = op.mg_level_matrix(level)
    bs = blocks.shape[2]
    G = np.zeros((op.E * bs, op.E * bs))
    for e in range(op.E):
        for s in range(nbr.shape[1]):
            t = nbr[e, s]
            if t >= 0:
                G[e * bs:(e + 1) * bs, t * bs:(t + 1) * bs] += blocks[e, s]
    return G


GALERKIN_CASES = [
    # kind, dim, n, degree, curved, strategy
    (POISSON, 2, 3, 4, True, "full"),
    (ELASTICITY, 2, 3, 4, True, "logarithmic"),
    (ELASTICITY, 3, 1, 3, True, "full"),
    (POISSON, 3, 2, 2, False, "twolevel"),
    (ELASTICITY, 2, 2, 1, False, "logarithmic"),  # degree-0 coarsest level
]


@pytest.mark.parametrize("case", GALERKIN_CASES, ids=lambda c: "k{}d{}n{}p{}c{}{}".format(*c))
def test_galerkin_levels_match_dense_triple_product(case):
    kind, dim, n, N, curved, strategy = case
    _, op, orc = product_and_oracle(kind, dim, n, N, curved, True)
    op.mg_setup(strategy=strategy)
    info = op.mg_info()
    degrees = info["degrees"]
    assert degrees == oracle.mg_levels(("twolevel", "logarithmic", "full").index(strategy), 1, N)
    P = prolongations(op, kind, dim, degrees)
    Al = dense(orc, op.ndof)
    for l in range(info["levels"] - 2, -1, -1):
        Al = P[l].T @ Al @ P[l]
        G = level_dense(op, l)
        assert np.abs(G - Al).max() <= 1e-12 * np.abs(Al).max(), l


def test_chebyshev_bounds_from_lanczos():
    kind, dim = ELASTICITY, 2
    _, op, orc = product_and_oracle(kind, dim, 3, 4, True, True)
    op.mg_setup(strategy="full")
    info = op.mg_info()
    P = prolongations(op, kind, dim, info["degrees"])
    A = [None] * len(P) + [dense(orc, op.ndof)]
    for l in range(len(P) - 1, -1, -1):
        A[l] = P[l].T @ A[l + 1] @ P[l]
    for l in range(1, info["levels"]):
        d = 1.0 / np.sqrt(np.diag(A[l]))
        lam = np.linalg.eigvalsh(d[:, None] * A[l] * d[None, :]).max()
        est = info["lambda_max"][l]
        assert 0.7 * lam <= est <= lam * (1 + 1e-9), (l, est, lam)


@pytest.mark.parametrize("coarse_space", ["dg", "p1"])
@pytest.mark.parametrize("case", [(POISSON, 2, 3, 4, "full"), (ELASTICITY, 2, 3, 4, "logarithmic"),
                                  (ELASTICITY, 3, 1, 3, "full"), (POISSON, 3, 2, 2, "twolevel")],
                         ids=lambda c: "k{}d{}n{}p{}{}".format(*c))
def test_vcycle_matches_dense_restatement(case, coarse_space):
    """coarse_space "p1": the restatement's coarsest level is the continuous P1 space of the
    mesh's own vertex numbering (the V-cycle does not depend on how the vertices are numbered)."""
    kind, dim, n, N, strategy = case
    m, op, orc = product_and_oracle(kind, dim, n, N, True, True)
    op.mg_setup(strategy=strategy, coarse_rtol=1e-13, coarse_max_it=20000, coarse_space=coarse_space)
    info = op.mg_info()
    P = prolongations(op, kind, dim, info["degrees"])
    lmax = list(info["lambda_max"])
    if coarse_space == "p1":
        P = [p1_embedding(m, op, kind, dim, info["degrees"][0])] + P
        lmax = [0.0] + lmax
    dm = DenseMultigrid(dense(orc, op.ndof), P, lmax, smooth_its=10, esteig=(0.01, 1.1))
    r = np.random.default_rng(5).standard_normal(op.ndof)
    z = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    op.mg_apply(dev(r), z)
    zr = dm.vcycle(r)
    assert np.abs(z.cpu().numpy() - zr).max() <= 1e-9 * np.abs(zr).max()


def _bj_iterations(op, b):
    op.set_preconditioner("bjacobi")
    op.bjacobi_setup(FP64)
    x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    return op.solve(dev(b), x, precision=FP64, rtol=1e-10)["iterations"]


@pytest.mark.parametrize("kind,dim,n", [(POISSON, 2, 8), (ELASTICITY, 2, 6), (ELASTICITY, 3, 2)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("coarse_space", ["dg", "p1"])
def test_mg_solve_reaches_target(kind, dim, n, precision, coarse_space):
    prec = FP64 if precision == "fp64" else MIXED
    _, op, orc = product_and_oracle(kind, dim, n, 4, True, True)
    _, _, _, f, g = mms_inputs(op, kind, dim, True)
    b = op.rhs(f, g)
    its_bj = _bj_iterations(op, b)
    op.mg_setup(smooth_precision=prec, coarse_space=coarse_space)
    op.set_preconditioner("mg")
    if prec == MIXED:
        op.bjacobi_setup(FP32)
    x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    st = op.solve(dev(b), x, precision=prec, rtol=1e-10, max_iterations=400)
    assert st["converged"] and st["rel_residual"] <= 1e-10, st
    assert np.linalg.norm(b - orc.apply(x.cpu().numpy())) / np.linalg.norm(b) <= 1.5e-10
    assert 3 * st["iterations"] <= its_bj, (st["iterations"], its_bj)


def test_mg_segmented_batch_and_multi_rhs():
    meshes = [make_mesh(2, n, 4, curved=True) for n in (5, 2, 4)]
    um, eoff = M.union(meshes)
    q = tandem_quadrature(2, 4)
    op = DGOperator(um, 4, ELASTICITY, q)
    orc = Oracle(um, 4, ELASTICITY, q)
    c0, c1 = material(ELASTICITY, 2, op.volume_coords(), True)
    op.set_material(c0, c1)
    orc.set_material(c0, c1)
    _, _, _, f, g = mms_inputs(op, ELASTICITY, 2, True)
    b = op.rhs(f, g)
    op.mg_setup()
    op.set_preconditioner("mg")
    x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    st, rel = solve_segmented(op, dev(b), x, eoff, precision=FP64, rtol=1e-10, max_iterations=400)
    assert st["converged"] and np.all(rel <= 1e-10), (st, rel)
    r = b - orc.apply(x.cpu().numpy())
    for i in range(len(meshes)):
        sl = slice(eoff[i] * op.bs, eoff[i + 1] * op.bs)
        assert np.linalg.norm(r[sl]) / np.linalg.norm(b[sl]) <= 1.5e-10
    # two right-hand sides with a padded leading dimension
    nrhs, ld = 2, op.ndof + 11
    B = torch.zeros(nrhs, ld, dtype=torch.float64, device=DEV)
    B[0, :op.ndof] = dev(b)
    B[1, :op.ndof] = dev(np.random.default_rng(2).standard_normal(op.ndof))
    X = torch.zeros(nrhs, ld, dtype=torch.float64, device=DEV)
    st = op.solve(B, X, precision=FP64, rtol=1e-10, nrhs=nrhs, ld=ld, max_iterations=400)
    assert st["converged"], st
    for k in range(nrhs):
        bk = B[k, :op.ndof].cpu().numpy()
        rk = bk - orc.apply(X[k, :op.ndof].cpu().numpy())
        assert np.linalg.norm(rk) / np.linalg.norm(bk) <= 1.5e-10


def test_mg_state_errors():
    _, op, _ = product_and_oracle(POISSON, 2, 3, 2, False, False)
    b = torch.ones(op.ndof, dtype=torch.float64, device=DEV)
    x = torch.zeros_like(b)
    op.set_preconditioner("mg")
    with pytest.raises(_ffi.TdgError, match="TDG_E_STATE"):
        op.solve(b, x)
    op.mg_setup()
    op.bjacobi_setup(FP32)
    with pytest.raises(_ffi.TdgError, match="TDG_E_INVALID"):
        op.solve(b, x, precision=FP32)
