"""One operator distributed over ranks (tandem_b200.partition) on CPU: the oracle (tandem's
element-centric apply) stands in for each rank's local operator, and gloo ranks exchange the ghost
blocks.

* Recursive coordinate bisection assigns every element, parts differ by at most one element.
* On every rank, the owned rows of the local operator (owned elements + one ghost layer, boundary
  codes and facet sides from the global mesh) and of the local right-hand side (volume and facet
  data sliced to the local elements and facets) equal the global rows to 1e-12, on a mesh with
  Dirichlet, natural, boundary-fault and interior-fault facets.
* With 2 and 3 gloo ranks: the exchange fills ghost blocks that start out zero (one vector, and two
  right-hand sides at a padded leading dimension whose padding it leaves alone), the distributed
  apply equals the global apply on the owned rows, and distributed block-Jacobi CG reaches the
  1e-10 relative residual of the global (oracle) operator."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cases import material, mms_inputs, tandem_quadrature
from oracle import Oracle
from tandem_b200 import mesh as M
from tandem_b200.partition import DistributedOperator, distributed_pcg, local_mesh, partition_elements


def _mesh(kind, dim, n, degree):
    """Top natural, left a fault (2D), other boundaries Dirichlet; an interior fault on x = 1/2 (2D)."""
    def boundary_bc(c):
        top = np.all(np.abs(c[:, :, dim - 1] - 1.0) < 1e-9, axis=1)
        left = np.all(np.abs(c[:, :, 0]) < 1e-9, axis=1)
        codes = np.where(top, M.BC_NATURAL, M.BC_DIRICHLET)
        return np.where(left & (dim == 2), M.BC_FAULT, codes)

    def interior_bc(c):
        on = np.all(np.abs(c[:, :, 0] - 0.5) < 1e-9, axis=1)
        return np.where(on & (dim == 2), M.BC_FAULT, M.BC_NONE)

    m = M.square_mesh(n) if dim == 2 else M.cube_mesh(n)
    return M.build(m, degree, boundary_bc=boundary_bc, interior_bc=interior_bc,
                   curve=M.box_boundary_surface(0.02))


def _setup(kind, dim, n, degree):
    m = _mesh(kind, dim, n, degree)
    q = tandem_quadrature(dim, degree)
    glob = Oracle(m, degree, kind, q)
    c0, c1 = material(kind, dim, glob.volume_coords(), True)
    glob.set_material(c0, c1)
    return m, q, glob, c0, c1


def _local_oracle(lm, degree, kind, q, c0, c1):
    orc = Oracle(lm.mesh, degree, kind, q)
    orc.set_material(c0[lm.elements], None if c1 is None else c1[lm.elements])
    return orc


@pytest.mark.parametrize("nparts", [1, 2, 3, 5, 8])
def test_partition_assigns_every_element_evenly(nparts):
    m = M.build(M.cube_mesh(3), 1)
    part = partition_elements(m, nparts)
    counts = np.bincount(part, minlength=nparts)
    assert counts.sum() == m.num_elements and len(counts) == nparts
    assert counts.max() - counts.min() <= 1


@pytest.mark.parametrize("kind,dim,n,degree,nparts", [(1, 2, 6, 3, 4), (0, 3, 2, 2, 2)])
def test_owned_rows_of_local_operators_equal_global_rows(kind, dim, n, degree, nparts):
    """In 2D the bisection cuts along the interior fault x = 1/2, so fault facets separate owned
    elements from ghosts and the slip terms depend on the local meshes keeping the global side
    order (with the sides in local order the owned right-hand side rows are off by 17 %)."""
    m, q, glob, c0, c1 = _setup(kind, dim, n, degree)
    bs = glob.ndof // m.num_elements
    x = np.random.default_rng(1).standard_normal(glob.ndof)
    y = glob.apply(x)
    _, _, _, f, g = mms_inputs(glob, kind, dim, True)
    g = g + 0.3 * np.cos(glob.facet_coords()[..., 0])[:, None, :]  # slip / Dirichlet data on every facet
    b = glob.rhs(f, g)
    part = partition_elements(m, nparts)
    up = m.facet_up
    on_cut = (m.facet_bc == M.BC_FAULT) & (up[:, 0] != up[:, 1]) & (part[up[:, 0]] != part[up[:, 1]])
    assert dim == 3 or on_cut.any()
    covered = np.zeros(m.num_elements, dtype=bool)
    for r in range(nparts):
        lm = local_mesh(m, part, r)
        assert np.all(part[lm.elements[:lm.n_owned]] == r) and np.all(part[lm.elements[lm.n_owned:]] != r)
        orc = _local_oracle(lm, degree, kind, q, c0, c1)
        xl = x.reshape(-1, bs)[lm.elements].ravel()
        yl = orc.apply(xl).reshape(-1, bs)[:lm.n_owned]
        ref = y.reshape(-1, bs)[lm.elements[:lm.n_owned]]
        assert np.abs(yl - ref).max() <= 1e-12 * np.abs(y).max()
        # right-hand side from sliced volume and facet data (Dirichlet and fault-slip terms
        # depend on each facet's side order, which the local mesh keeps)
        bl = orc.rhs(f[lm.elements], g[lm.facets]).reshape(-1, bs)[:lm.n_owned]
        bref = b.reshape(-1, bs)[lm.elements[:lm.n_owned]]
        assert np.abs(bl - bref).max() <= 1e-12 * np.abs(b).max()
        covered[lm.elements[:lm.n_owned]] = True
    assert covered.all()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _dd_worker(rank, world, port, q, kind, dim, n, degree):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        m, quad, glob, c0, c1 = _setup(kind, dim, n, degree)
        bs = glob.ndof // m.num_elements
        lm = local_mesh(m, partition_elements(m, world), rank)
        orc = _local_oracle(lm, degree, kind, quad, c0, c1)

        def apply_local(x, y):
            y.copy_(torch.from_numpy(orc.apply(x.numpy())))

        A = DistributedOperator(lm, bs, apply_local)
        own = lm.elements[:lm.n_owned]
        # the exchange fills ghost blocks that start at zero
        xg = np.random.default_rng(7).standard_normal(glob.ndof)
        xl = torch.zeros(A.n_local, dtype=torch.float64)
        xl[:A.n_owned] = torch.from_numpy(xg.reshape(-1, bs)[own].ravel())
        y = torch.zeros_like(xl)
        A.apply(xl, y)
        ghosts_ok = np.array_equal(xl.numpy().reshape(-1, bs)[lm.n_owned:], xg.reshape(-1, bs)[lm.elements[lm.n_owned:]])
        # two right-hand sides at a padded leading dimension: ghosts filled, padding untouched
        ld = A.n_local + 5
        X = torch.full((2, ld), -1.0, dtype=torch.float64)
        X[0, :A.n_local] = 0.0
        X[1, :A.n_local] = 0.0
        X[0, :A.n_owned] = torch.from_numpy(xg.reshape(-1, bs)[own].ravel())
        X[1, :A.n_owned] = 2.0 * X[0, :A.n_owned]
        A.halo.exchange(X.reshape(-1), nrhs=2, ld=ld)
        gl = xg.reshape(-1, bs)[lm.elements[lm.n_owned:]].ravel()
        ghosts_ok = ghosts_ok and np.array_equal(X[0, A.n_owned:A.n_local].numpy(), gl) \
            and np.array_equal(X[1, A.n_owned:A.n_local].numpy(), 2.0 * gl) and bool(torch.all(X[:, A.n_local:] == -1.0))
        ref = glob.apply(xg).reshape(-1, bs)[own]
        apply_err = float(np.abs(y.numpy().reshape(-1, bs)[:lm.n_owned] - ref).max() / np.abs(ref).max())
        # distributed block-Jacobi CG on the manufactured problem
        _, _, _, f, g = mms_inputs(glob, kind, dim, True)
        bg = glob.rhs(f, g)
        b = torch.zeros(A.n_local, dtype=torch.float64)
        b[:A.n_owned] = torch.from_numpy(bg.reshape(-1, bs)[own].ravel())
        inv = np.linalg.inv(orc.assemble_diag()[:lm.n_owned])

        def precondition(r, z):
            rr = r.numpy()[:A.n_owned].reshape(-1, bs)
            z[:A.n_owned] = torch.from_numpy(np.einsum("eij,ej->ei", inv, rr).ravel())

        x = torch.zeros_like(b)
        st = distributed_pcg(A, precondition, b, x, rtol=1e-10, max_iterations=5000)
        parts = [None] * world
        dist.all_gather_object(parts, (own, x.numpy()[:A.n_owned].reshape(-1, bs)))
        rel = None
        if rank == 0:
            xs = np.zeros((m.num_elements, bs))
            for o, v in parts:
                xs[o] = v
            rel = float(np.linalg.norm(bg - glob.apply(xs.ravel())) / np.linalg.norm(bg))
        q.put((rank, ghosts_ok, apply_err, st, rel))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind,dim,n,degree,world", [(1, 2, 6, 3, 2), (0, 3, 2, 2, 3)])
def test_distributed_apply_and_pcg_gloo(kind, dim, n, degree, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dd_worker, args=(r, world, port, q, kind, dim, n, degree)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, ghosts_ok, apply_err, st, rel in res:
        assert ghosts_ok, rank
        assert apply_err <= 1e-12, (rank, apply_err)
        assert st["converged"], (rank, st)
        if rank == 0:
            assert rel <= 1.5e-10, rel
