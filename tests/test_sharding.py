"""Multi-rank work distribution on CPU ranks (gloo, world size 2): column blocks of the Green's
function, LPT assignment of uneven problems, gather of column blocks to rank 0, and a rank that
fails between steps being detected on the host by the others (short process-group timeout)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from tandem_b200.sharding import column_block, gather_columns, lpt_assign


def test_column_blocks_partition():
    for ncols in (1, 7, 1280):
        for world in (1, 2, 3, 8):
            blocks = [column_block(ncols, world, r) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == ncols
            assert all(blocks[i][1] == blocks[i + 1][0] for i in range(world - 1))
            sizes = [e - s for s, e in blocks]
            assert max(sizes) - min(sizes) <= 1


def test_lpt_balances_uneven_problems():
    rng = np.random.default_rng(0)
    costs = np.exp(rng.uniform(np.log(1e3), np.log(4e4), size=48))
    parts = lpt_assign(costs, 4)
    assert sorted(i for p in parts for i in p) == list(range(48))
    loads = [costs[p].sum() for p in parts]
    # LPT is within 4/3 of optimal; the mean load is a lower bound of the optimum
    assert max(loads) <= 4 / 3 * max(costs.sum() / 4, costs.max()) + 1e-9


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gather_worker(rank, world, port, ncols, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    s, e = column_block(ncols, world, rank)
    local = torch.arange(s, e, dtype=torch.float64).repeat(3, 1) + 1000 * torch.arange(3.0)[:, None]
    out = gather_columns(local, ncols)
    if rank == 0:
        q.put(out.numpy())
    dist.destroy_process_group()


def test_gather_columns_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ncols = 11
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, ncols, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = q.get(timeout=60)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = np.arange(ncols, dtype=float)[None, :] + 1000 * np.arange(3.0)[:, None]
    np.testing.assert_array_equal(out, ref)


def _failing_worker(rank, world, port, q):
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
    t = torch.ones(4)
    dist.all_reduce(t)  # step 1: both ranks
    if rank == 1:
        os._exit(0)  # rank 1 leaves between steps, with nothing in flight
    try:
        dist.all_reduce(t)  # step 2: rank 0 must learn of it through an error, not hang
        q.put("no error")
    except Exception as e:  # noqa: BLE001
        q.put(type(e).__name__)


def test_rank_failure_detected_by_timeout():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert res != "no error"


def test_uneven_batch_share_reproduces_its_problems():
    """A rank's share of the uneven batch (workloads.uneven_batch(problems=...)) holds exactly the
    listed problems of the full batch: same meshes, material and force, in the listed order."""
    from cases import tandem_quadrature
    from tandem_b200.sharding import lpt_assign
    from tandem_b200.workloads import uneven_batch, uneven_batch_cells
    q = tandem_quadrature(2, 2)
    full = uneven_batch(6, 2, q, lo=20, hi=200)
    cells = uneven_batch_cells(6, lo=20, hi=200)
    shares = lpt_assign(2 * cells ** 2, 2)
    assert sorted(shares[0] + shares[1]) == list(range(6))
    for share in shares:
        part = uneven_batch(6, 2, q, lo=20, hi=200, problems=share)
        assert part.op.E == sum(int(full.sizes[i]) for i in share)
        for j, i in enumerate(share):
            a = slice(full.elem_offsets[i], full.elem_offsets[i + 1])
            b = slice(part.elem_offsets[j], part.elem_offsets[j + 1])
            np.testing.assert_array_equal(part.force[b], full.force[a])
            np.testing.assert_array_equal(part.op.material_nodal(0)[b], full.op.material_nodal(0)[a])
            np.testing.assert_array_equal(part.mesh.geo_nodes[b], full.mesh.geo_nodes[a])
