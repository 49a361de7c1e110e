"""Device apply, block Jacobi and solve against the oracle (CPU restatement of tandem).

Tolerances: FP64 results agree with the oracle to 1e-12 relative (max-norm over the vector,
summation order differs); FP32 applies to 2e-5 relative; solutions to the relative residual
target 1e-10 of the metric."""
import math

import numpy as np
import pytest
import torch

from cases import make_mesh, mms_inputs, product_and_oracle, tandem_quadrature
from oracle import Oracle
from tandem_b200 import _ffi
from tandem_b200 import mesh as M
from tandem_b200.operator import DGOperator, ELASTICITY, FP32, FP64, POISSON

pytestmark = pytest.mark.gpu
DEV = "cuda:0"

CASES = [
    # kind, dim, n, degree, curved, variable
    (POISSON, 2, 4, 4, False, False),
    (POISSON, 2, 3, 1, True, True),
    (POISSON, 2, 3, 2, True, True),
    (POISSON, 2, 3, 3, False, True),
    (POISSON, 3, 2, 4, True, True),
    (POISSON, 3, 2, 2, False, True),
    (ELASTICITY, 2, 3, 4, True, True),
    (ELASTICITY, 2, 3, 1, False, False),
    (ELASTICITY, 3, 2, 4, True, True),
    (ELASTICITY, 3, 2, 3, True, True),
    (ELASTICITY, 3, 1, 1, False, True),
]


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def dev(x, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=DEV)


@pytest.mark.parametrize("case", CASES, ids=lambda c: "k{}d{}n{}p{}c{}v{}".format(*c))
def test_apply_fp64_matches_oracle(case):
    kind, dim, n, N, curved, var = case
    _, op, orc = product_and_oracle(kind, dim, n, N, curved, var)
    x = np.random.default_rng(7).standard_normal(op.ndof)
    y = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    op.apply(dev(x), y)
    torch.cuda.synchronize()
    assert rel(y.cpu().numpy(), orc.apply(x)) < 1e-12


@pytest.mark.parametrize("case", CASES[::2], ids=lambda c: "k{}d{}n{}p{}c{}v{}".format(*c))
def test_apply_fp32_close_to_oracle(case):
    kind, dim, n, N, curved, var = case
    _, op, orc = product_and_oracle(kind, dim, n, N, curved, var)
    x = np.random.default_rng(8).standard_normal(op.ndof)
    y = torch.zeros(op.ndof, dtype=torch.float32, device=DEV)
    op.apply(dev(x, torch.float32), y, precision=FP32)
    torch.cuda.synchronize()
    ref = orc.apply(x.astype(np.float32).astype(np.float64))
    assert np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref) < 2e-5


def test_multi_rhs_apply_equals_single():
    _, op, orc = product_and_oracle(ELASTICITY, 3, 2, 4, True, True)
    nrhs, ld = 3, op.ndof + 37
    X = torch.randn(nrhs, ld, dtype=torch.float64, device=DEV)
    Y = torch.zeros(nrhs, ld, dtype=torch.float64, device=DEV)
    op.apply(X, Y, nrhs=nrhs, ld=ld)
    for r in range(nrhs):
        y = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
        op.apply(X[r, :op.ndof].contiguous(), y)
        assert torch.equal(y, Y[r, :op.ndof])
        assert torch.all(Y[r, op.ndof:] == 0)


@pytest.mark.parametrize("kind,dim,curved", [(POISSON, 2, False), (ELASTICITY, 2, True), (ELASTICITY, 3, True),
                                              (POISSON, 3, True)])
def test_block_jacobi_blocks_and_apply(kind, dim, curved):
    _, op, orc = product_and_oracle(kind, dim, 3 if dim == 2 else 2, 4, curved, True)
    op.bjacobi_setup(FP64)
    blocks = op.bjacobi_blocks()
    ref = orc.assemble_diag()
    assert rel(blocks, ref) < 1e-12
    r = np.random.default_rng(3).standard_normal(op.ndof)
    z = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    op.bjacobi_apply(dev(r), z)
    torch.cuda.synchronize()
    zr = np.concatenate([np.linalg.solve(ref[e], r[e * op.bs:(e + 1) * op.bs]) for e in range(op.E)])
    assert rel(z.cpu().numpy(), zr) < 1e-10
    op.bjacobi_setup(FP32)
    z32 = torch.zeros(op.ndof, dtype=torch.float32, device=DEV)
    op.bjacobi_apply(dev(r, torch.float32), z32, precision=FP32)
    torch.cuda.synchronize()
    assert np.linalg.norm(z32.cpu().numpy() - zr) / np.linalg.norm(zr) < 1e-4


def test_not_spd_block_is_reported():
    m = make_mesh(2, 2, 2)
    op = DGOperator(m, 2, ELASTICITY, tandem_quadrature(2, 2))
    X = op.volume_coords()
    op.set_material(2.0 * np.ones(X.shape[:2]), -np.ones(X.shape[:2]))
    with pytest.raises(_ffi.TdgError, match="TDG_E_NOT_SPD"):
        op.bjacobi_setup(FP64)


@pytest.mark.parametrize("kind,dim,n,curved", [(POISSON, 2, 8, False), (ELASTICITY, 2, 4, True),
                                                (ELASTICITY, 3, 2, True)])
@pytest.mark.parametrize("precision", [FP64, FP32])
def test_solve_matches_oracle(kind, dim, n, curved, precision):
    m, op, orc = product_and_oracle(kind, dim, n, 4, curved, True)
    sc, c0, c1, f, g = mms_inputs(op, kind, dim, True)
    b = op.rhs(f, g)
    xo, st_o = orc.cg(b, rtol=1e-12)
    op.bjacobi_setup(precision)
    x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    st = op.solve(dev(b), x, precision=precision, rtol=1e-10)
    assert st["converged"] and st["rel_residual"] <= 1e-10, st
    xs = x.cpu().numpy()
    # true FP64 residual through the oracle
    assert np.linalg.norm(b - orc.apply(xs)) / np.linalg.norm(b) <= 1.5e-10
    assert np.linalg.norm(xs - xo) / np.linalg.norm(xo) < 1e-7


def test_config1_full_size_apply():
    """configs[0] at full size: 64 x 64 x 2 triangles, degree 4, 122,880 DOF."""
    m = make_mesh(2, 64, 4)
    q = tandem_quadrature(2, 4)
    op = DGOperator(m, 4, POISSON, q)
    orc = Oracle(m, 4, POISSON, q)
    K = np.ones((op.E, op.Nq))
    op.set_material(K)
    orc.set_material(K)
    x = np.random.default_rng(11).standard_normal(op.ndof)
    y = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    op.apply(dev(x), y)
    torch.cuda.synchronize()
    assert rel(y.cpu().numpy(), orc.apply(x)) < 1e-12


def test_elasticity_3d_properties_at_scale():
    """Size-independent properties on a 12^3 x 6 curved mesh (10,368 tets, 1.1 M DOF): symmetry
    x.Ay = y.Ax, translations annihilated up to boundary terms only, and a slice of elements
    against the oracle."""
    m = make_mesh(3, 12, 4, True)
    q = tandem_quadrature(3, 4)
    op = DGOperator(m, 4, ELASTICITY, q)
    orc = Oracle(m, 4, ELASTICITY, q)
    from cases import material
    c0, c1 = material(ELASTICITY, 3, op.volume_coords(), True, ell=0.2)
    op.set_material(c0, c1)
    orc.set_material(c0, c1)
    g = torch.Generator(device=DEV).manual_seed(5)
    x = torch.randn(op.ndof, dtype=torch.float64, device=DEV, generator=g)
    z = torch.randn(op.ndof, dtype=torch.float64, device=DEV, generator=g)
    ax = torch.empty_like(x)
    az = torch.empty_like(x)
    op.apply(x, ax)
    op.apply(z, az)
    torch.cuda.synchronize()
    s1, s2 = torch.dot(z, ax).item(), torch.dot(x, az).item()
    assert abs(s1 - s2) <= 1e-12 * (torch.norm(z) * torch.norm(ax)).item()
    xn = x.cpu().numpy()
    yref = np.zeros(op.ndof)
    e0, e1 = 3000, 3400
    orc.apply_range(e0, e1, xn, yref)
    bs = op.bs
    assert rel(ax.cpu().numpy()[e0 * bs:e1 * bs], yref[e0 * bs:e1 * bs]) < 1e-12


@pytest.mark.parametrize("precision", [FP64, FP32])
def test_segmented_solve_of_a_mesh_union(precision):
    """Three independent 2D elasticity problems of different sizes in one block-diagonal operator:
    each problem's solution equals its own solve."""
    from tandem_b200.operator import solve_segmented
    from cases import material
    meshes = [make_mesh(2, n, 4, curved=True) for n in (2, 5, 3)]
    um, eoff = M.union(meshes)
    q = tandem_quadrature(2, 4)
    op = DGOperator(um, 4, ELASTICITY, q)
    orc = Oracle(um, 4, ELASTICITY, q)
    c0, c1 = material(ELASTICITY, 2, op.volume_coords(), True)
    op.set_material(c0, c1)
    orc.set_material(c0, c1)
    _, _, _, f, g = mms_inputs(op, ELASTICITY, 2, True)
    b = op.rhs(f, g)
    op.bjacobi_setup(precision)
    x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    st, rel = solve_segmented(op, dev(b), x, eoff, precision=precision, rtol=1e-10)
    assert st["converged"] and np.all(rel <= 1e-10), (st, rel)
    xs = x.cpu().numpy()
    bs = op.bs
    r = b - orc.apply(xs)
    for i in range(len(meshes)):
        sl = slice(eoff[i] * bs, eoff[i + 1] * bs)
        assert np.linalg.norm(r[sl]) / np.linalg.norm(b[sl]) <= 1.5e-10


@pytest.mark.parametrize("precision", ["mixed", FP32])
def test_segmented_solve_keeps_each_problem_recurrence(precision):
    """Problems of very different size in one segmented solve: a reliable update asked for by one
    problem replaces only that problem's residual, so no problem's Krylov space is restarted by
    the others.  Every problem converges, and the segmented solve needs at most 25% (+16) more
    iterations than the slowest problem solved alone."""
    from tandem_b200.operator import MIXED, solve_segmented
    from cases import material
    prec = MIXED if precision == "mixed" else precision
    sizes = (14, 3, 9, 2, 6)
    meshes = [make_mesh(2, n, 4, curved=True) for n in sizes]
    q = tandem_quadrature(2, 4)

    def problem(m):
        op = DGOperator(m, 4, ELASTICITY, q)
        op.set_material(*material(ELASTICITY, 2, op.volume_coords(), True, ell=0.3))
        _, _, _, f, g = mms_inputs(op, ELASTICITY, 2, True)
        op.bjacobi_setup(FP32)
        return op, op.rhs(f, g)

    alone = []
    for m in meshes:
        op, b = problem(m)
        x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
        alone.append(op.solve(dev(b), x, precision=prec, rtol=1e-10, max_iterations=20000)["iterations"])
    um, eoff = M.union(meshes)
    op, b = problem(um)
    orc = Oracle(um, 4, ELASTICITY, q)
    orc.set_material(*material(ELASTICITY, 2, op.volume_coords(), True, ell=0.3))
    x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    st, relr = solve_segmented(op, dev(b), x, eoff, precision=prec, rtol=1e-10, max_iterations=20000)
    assert st["converged"] and np.all(relr <= 1e-10), (st, relr)
    assert st["iterations"] <= 1.25 * max(alone) + 16, (st["iterations"], alone)
    r = b - orc.apply(x.cpu().numpy())
    bs = op.bs
    for i in range(len(meshes)):
        sl = slice(eoff[i] * bs, eoff[i + 1] * bs)
        assert np.linalg.norm(r[sl]) / np.linalg.norm(b[sl]) <= 1.5e-10


@pytest.mark.parametrize("case", CASES[::3], ids=lambda c: "k{}d{}n{}p{}c{}v{}".format(*c))
def test_apply_mixed_fp64_vectors(case):
    """TDG_MIXED: FP32 tensor-core arithmetic on FP64 vectors agrees with the oracle to FP32
    accuracy (2e-5 relative, as the FP32 apply) and with the FP32-vector apply of the same rounded
    input to 1e-6 (same kernel, only the vector type differs)."""
    from tandem_b200.operator import MIXED
    kind, dim, n, N, curved, var = case
    _, op, orc = product_and_oracle(kind, dim, n, N, curved, var)
    x = np.random.default_rng(9).standard_normal(op.ndof)
    xr = x.astype(np.float32).astype(np.float64)
    y = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    op.apply(dev(xr), y, precision=MIXED)
    y32 = torch.zeros(op.ndof, dtype=torch.float32, device=DEV)
    op.apply(dev(xr, torch.float32), y32, precision=FP32)
    torch.cuda.synchronize()
    ref = orc.apply(xr)
    got = y.cpu().numpy()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-5
    assert np.linalg.norm(got - y32.double().cpu().numpy()) / np.linalg.norm(ref) < 1e-6


@pytest.mark.parametrize("kind,dim,n,curved", [(POISSON, 2, 8, False), (ELASTICITY, 3, 2, True)])
def test_mixed_solve_reaches_fp64_target(kind, dim, n, curved):
    from tandem_b200.operator import MIXED
    m, op, orc = product_and_oracle(kind, dim, n, 4, curved, True)
    sc, c0, c1, f, g = mms_inputs(op, kind, dim, True)
    b = op.rhs(f, g)
    op.bjacobi_setup(MIXED)
    x = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    st = op.solve(dev(b), x, precision=MIXED, rtol=1e-10)
    assert st["converged"] and st["rel_residual"] <= 1e-10, st
    xs = x.cpu().numpy()
    assert np.linalg.norm(b - orc.apply(xs)) / np.linalg.norm(b) <= 1.5e-10


@pytest.mark.parametrize("case", CASES, ids=lambda c: "k{}d{}n{}p{}c{}v{}".format(*c))
@pytest.mark.parametrize("ctas", [1, 2])
@pytest.mark.parametrize("family", ["face", "face2"])
def test_apply_face_centric_matches_oracle(case, ctas, family):
    """Face-centric FP64 apply (volume kernel + one pass over the facets with atomics; face2: the
    software-pipelined pair) against the oracle, 1e-12 like the element-centric kernel."""
    kind, dim, n, N, curved, var = case
    _, op, orc = product_and_oracle(kind, dim, n, N, curved, var)
    op.set_apply_config(FP64, family, ctas)
    x = np.random.default_rng(7).standard_normal(op.ndof)
    y = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    op.apply(dev(x), y)
    torch.cuda.synchronize()
    assert rel(y.cpu().numpy(), orc.apply(x)) < 1e-12


@pytest.mark.parametrize("family", ["face", "face2"])
def test_face_centric_multi_rhs_and_solve(family):
    _, op, orc = product_and_oracle(ELASTICITY, 3, 2, 4, True, True)
    op.set_apply_config(FP64, family)
    nrhs, ld = 3, op.ndof + 37
    X = torch.randn(nrhs, ld, dtype=torch.float64, device=DEV)
    Y = torch.full((nrhs, ld), 7.0, dtype=torch.float64, device=DEV)
    op.apply(X, Y, nrhs=nrhs, ld=ld)
    for r in range(nrhs):
        y = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
        op.apply(X[r, :op.ndof].contiguous(), y)
        scale = torch.max(torch.abs(y)).item()
        assert torch.max(torch.abs(y - Y[r, :op.ndof])).item() <= 1e-14 * scale
        assert torch.all(Y[r, op.ndof:] == 7.0)


@pytest.mark.parametrize("case", CASES, ids=lambda c: "k{}d{}n{}p{}c{}v{}".format(*c))
def test_face2_points_per_pass_matches_oracle(case):
    """The pipelined FP64 pair with its volume term in several passes over the quadrature points
    (tdg_set_apply_tile: every pass height from one step up to the first at or above the point count)
    against the oracle, 1e-12 like the one-pass layout."""
    kind, dim, n, N, curved, var = case
    _, op, orc = product_and_oracle(kind, dim, n, N, curved, var)
    x = np.random.default_rng(7).standard_normal(op.ndof)
    ref = orc.apply(x)
    step = 8 if dim == 3 else 4
    heights = list(range(step, op.Nq + step, step))
    assert len(heights) >= 1 and heights[-1] >= op.Nq
    for tile in heights:
        op.set_apply_config(FP64, "face2", 2, tile)
        y = torch.full((op.ndof,), 3.0, dtype=torch.float64, device=DEV)
        op.apply(dev(x), y)
        torch.cuda.synchronize()
        assert rel(y.cpu().numpy(), ref) < 1e-12, tile


def test_face2_points_per_pass_arguments_and_autotune():
    """Pass heights off the step, negative or for FP32 are refused; the autotuner times the
    pipelined pair at the heights that cover the points in 1 to 4 passes and keeps a working pick."""
    _, op, orc = product_and_oracle(ELASTICITY, 3, 2, 4, True, True)
    for bad in (-8, 4, 12, 57):
        with pytest.raises(RuntimeError):
            op.set_apply_config(FP64, "face2", 2, bad)
    with pytest.raises(RuntimeError):
        op.set_apply_config(FP32, "tc05", 2, 8)
    tune = op.autotune(FP64)
    tiles = sorted({e["tile"] for e in tune if e["family"] == "face2"})
    step = 8
    heights = {math.ceil(math.ceil(op.Nq / p) / step) * step for p in (2, 3, 4)}
    want = [0] + sorted(h for h in heights if h < op.Nq)
    assert tiles == want, (tiles, op.Nq)
    assert all(e["tile"] == 0 for e in tune if e["family"] != "face2")
    x = np.random.default_rng(3).standard_normal(op.ndof)
    y = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    op.apply(dev(x), y)
    torch.cuda.synchronize()
    assert rel(y.cpu().numpy(), orc.apply(x)) < 1e-12


@pytest.mark.parametrize("family", ["face", "tc05"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "k{}d{}n{}p{}c{}v{}".format(*c))
def test_apply_face_centric_fp32_and_mixed(case, family):
    """Face-centric FP32 kernels (3xTF32; family tc05 with the volume term on tcgen05.mma and
    tensor memory) on FP32 and on FP64 vectors (mixed) against the oracle to FP32 accuracy (2e-5,
    as the element-centric FP32 apply)."""
    from tandem_b200.operator import MIXED
    kind, dim, n, N, curved, var = case
    _, op, orc = product_and_oracle(kind, dim, n, N, curved, var)
    op.set_apply_config(FP32, family)
    x = np.random.default_rng(12).standard_normal(op.ndof)
    xr = x.astype(np.float32).astype(np.float64)
    ref = orc.apply(xr)
    y32 = torch.zeros(op.ndof, dtype=torch.float32, device=DEV)
    op.apply(dev(xr, torch.float32), y32, precision=FP32)
    ym = torch.zeros(op.ndof, dtype=torch.float64, device=DEV)
    op.apply(dev(xr), ym, precision=MIXED)
    torch.cuda.synchronize()
    for got in (y32.double().cpu().numpy(), ym.cpu().numpy()):
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-5


@pytest.mark.parametrize("family", ["face", "tc05"])
@pytest.mark.parametrize("kind,dim,N", [(ELASTICITY, 3, 4), (POISSON, 3, 3), (ELASTICITY, 2, 4)])
def test_fp32_face_families_multi_rhs_padded(family, kind, dim, N):
    """The FP32 face-centric families (tc05: the tcgen05 volume kernel) on three right-hand sides at
    a padded leading dimension, FP32 and mixed vectors: every column matches its own single-vector
    apply to FP32 rounding (1e-6 relative; the facet atomics may add in another order) and the
    padding is left untouched."""
    from tandem_b200.operator import MIXED
    _, op, orc = product_and_oracle(kind, dim, 2, N, True, True)
    op.set_apply_config(FP32, family)
    nrhs, ld = 3, op.ndof + 37
    for prec, dt in ((FP32, torch.float32), (MIXED, torch.float64)):
        X = torch.randn(nrhs, ld, dtype=dt, device=DEV)
        Y = torch.full((nrhs, ld), 7.0, dtype=dt, device=DEV)
        op.apply(X, Y, precision=prec, nrhs=nrhs, ld=ld)
        for r in range(nrhs):
            y = torch.zeros(op.ndof, dtype=dt, device=DEV)
            op.apply(X[r, :op.ndof].contiguous(), y, precision=prec)
            scale = torch.max(torch.abs(y)).item()
            assert torch.max(torch.abs(y - Y[r, :op.ndof])).item() <= 1e-6 * scale
            assert torch.all(Y[r, op.ndof:] == 7.0)
