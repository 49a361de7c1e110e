"""Work distribution across ranks (one process per GPU, torch.distributed).

The operator apply itself needs no collective on one mesh per GPU.  The two batched workloads
shard without any data-path exchange:
  * Green's functions: independent right-hand sides (fault basis coefficients) -> contiguous
    column blocks per rank, one gather of the column blocks to rank 0 at the end
    (tandem computes the columns in sequence, app/form/SeasQDDiscreteGreenOperator.cpp:519-574);
  * uneven problem batches: independent meshes -> longest-processing-time-first assignment by
    element count.
"""
from __future__ import annotations

import heapq

import numpy as np


def column_block(ncols: int, world: int, rank: int) -> tuple[int, int]:
    """[start, stop) of the columns of `rank` (blocks differ by at most one column)."""
    base, extra = divmod(ncols, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def lpt_assign(costs, world: int) -> list[list[int]]:
    """Longest-processing-time-first: problems in decreasing cost go to the least loaded rank.
    Returns per-rank lists of problem indices (each sorted)."""
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in np.argsort(-np.asarray(costs, dtype=float), kind="stable"):
        load, r = heapq.heappop(heap)
        out[r].append(int(i))
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(x) for x in out]


def gather_columns(local, ncols: int, group=None):
    """Gathers the column blocks [rows, start:stop) of every rank into a [rows, ncols] tensor on
    rank 0 (None elsewhere).  Works with the gloo (CPU tensors) and nccl (CUDA tensors) backends."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    rows = local.shape[0]
    width = max(column_block(ncols, world, r)[1] - column_block(ncols, world, r)[0] for r in range(world))
    buf = torch.zeros(rows, width, dtype=local.dtype, device=local.device)
    buf[:, :local.shape[1]] = local
    parts = [torch.zeros_like(buf) for _ in range(world)] if rank == 0 else None
    dist.gather(buf, parts, dst=0, group=group)
    if rank != 0:
        return None
    out = torch.zeros(rows, ncols, dtype=local.dtype, device=local.device)
    for r in range(world):
        s, e = column_block(ncols, world, r)
        out[:, s:e] = parts[r][:, :e - s]
    return out
