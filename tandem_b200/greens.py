"""Discrete Green's function operator of a fault: tandem's SeasQDDiscreteGreenOperator core
(app/form/SeasQDDiscreteGreenOperator.cpp) on the device.

* ``compute``: the columns G[:, i] = traction(solve(rhs(slip = e_i))) in batched multi-RHS solves
  (tandem: partial_assemble_discrete_greens_function, :493-578, one KSPSolve per column), with an
  optional checkpoint after every batch;
* ``compute_boundary_traction``: the traction of the zero-slip solve with the boundary / body data
  at time 1 (compute_boundary_traction, :129-150);
* ``update_traction``: traction = G S + time t_boundary (update_traction, :115-127) as one kernel
  of the library (tdg_gf_traction_update) over any number of slip states;
* ``save`` / ``load``: a checkpoint that does not depend on how the fault was partitioned or
  ordered (write_discrete_greens_operator / load_discrete_greens_operator, :201-237, :432-491):
  G is stored with the global facet labels of its block rows and columns and the set of computed
  columns; loading into a different facet order permutes rows and columns by label (tandem
  permutes by its facet-label index set when the communicator size changed).  Files are written
  to `path.tmp` and renamed, the previous checkpoint kept as `path.bu` (tandem's back_up_file).
"""
from __future__ import annotations

import os

import numpy as np

from .operator import FP64, DGOperator, Fault

_FORMAT = 1


def save_checkpoint(path: str, G: np.ndarray, done: np.ndarray, labels: np.ndarray, nbf: int) -> None:
    """Writes G [n, n] (only computed columns are meaningful), done [n] and the facet labels of the
    block rows / columns (n = len(labels) * nbf)."""
    labels = np.asarray(labels, dtype=np.int64)
    n = len(labels) * nbf
    if G.shape != (n, n) or done.shape != (n,):
        raise ValueError("G / done do not match labels x nbf")
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        np.savez(f, format=np.int64(_FORMAT), G=np.ascontiguousarray(G, dtype=np.float64),
                 done=done.astype(bool), labels=labels, nbf=np.int64(nbf))
    if os.path.exists(path):
        os.replace(path, path + ".bu")
    os.replace(tmp, path)


def load_checkpoint(path: str, labels: np.ndarray, nbf: int) -> tuple[np.ndarray, np.ndarray]:
    """Reads a checkpoint into the block order given by `labels`; returns (G, done)."""
    labels = np.asarray(labels, dtype=np.int64)
    with np.load(path) as z:
        if int(z["format"]) != _FORMAT:
            raise ValueError("unknown checkpoint format")
        if int(z["nbf"]) != nbf:
            raise ValueError(f"checkpoint has {int(z['nbf'])} basis functions per facet, expected {nbf}")
        old = z["labels"]
        if len(old) != len(labels) or not np.array_equal(np.sort(old), np.sort(labels)):
            raise ValueError("checkpoint was written for a different set of fault facets")
        G_old, done_old = z["G"], z["done"]
    pos = {int(l): i for i, l in enumerate(labels)}
    blk = np.array([pos[int(l)] for l in old])                   # old block -> new block
    idx = (blk[:, None] * nbf + np.arange(nbf)[None, :]).ravel()  # old index -> new index
    n = len(labels) * nbf
    G = np.zeros((n, n))
    G[np.ix_(idx, idx)] = G_old
    done = np.zeros(n, dtype=bool)
    done[idx] = done_old
    return G, done


class DiscreteGreensOperator:
    """G (FP64, on the device) of `fault` over operator `op`; `labels` are the global ids of the
    fault facets in the order of the fault's basis (default: the facet ids themselves)."""

    def __init__(self, op: DGOperator, fault: Fault, labels=None):
        import torch
        self.op, self.fault = op, fault
        self.labels = np.asarray(fault._facets if labels is None else labels, dtype=np.int64)
        if len(self.labels) != fault.nfault:
            raise ValueError("one label per fault facet")
        self.n = fault.ncoef
        self.G = torch.zeros(self.n, self.n, dtype=torch.float64, device="cuda")
        self.done = np.zeros(self.n, dtype=bool)
        self.t_boundary = torch.zeros(self.n, dtype=torch.float64, device="cuda")
        self.stats: list[dict] = []

    @property
    def current(self) -> int:
        return int(self.done.sum())

    def compute(self, precision: int = FP64, rtol: float = 1e-10, batch: int = 256, checkpoint: str | None = None,
                max_batches: int | None = None, **solve_kw) -> None:
        """Solves the columns not computed yet, `batch` right-hand sides per solve; writes the
        checkpoint after every batch.  max_batches bounds the batches of this call."""
        from .operator import greens_function
        todo = np.nonzero(~self.done)[0]
        for b, s in enumerate(range(0, len(todo), batch)):
            if max_batches is not None and b >= max_batches:
                break
            cols = todo[s:s + batch]
            G, st = greens_function(self.op, self.fault, precision=precision, rtol=rtol, columns=cols,
                                    batch=len(cols), **solve_kw)
            import torch
            self.G[:, torch.as_tensor(cols, device="cuda")] = G
            self.done[cols] = True
            self.stats.extend(st)
            if checkpoint:
                self.save(checkpoint)

    def compute_boundary_traction(self, force_Q=None, bc_q=None, precision: int = FP64, rtol: float = 1e-10,
                                  **solve_kw) -> None:
        """t_boundary = traction of the solve with zero slip and the given body force / boundary
        data (evaluated at time 1)."""
        import torch
        b = torch.as_tensor(self.op.rhs(force_Q, bc_q), device="cuda")
        x = torch.zeros_like(b)
        self.op.solve(b, x, precision=precision, rtol=rtol, **solve_kw)
        slip = torch.zeros(self.n, dtype=torch.float64, device="cuda")
        out = torch.empty(self.n, dtype=torch.float64, device="cuda")
        self.fault.traction(x, slip, out)
        self.t_boundary = out

    def update_traction(self, slip, time: float = 0.0, stream=None):
        """traction = G slip + time t_boundary for slip [n] or [n, k] (k slip states at once), one
        kernel of the library (tdg_gf_traction_update: G read once per group of 4 states, the
        boundary term fused)."""
        import ctypes as C
        import torch
        from . import _ffi
        from .operator import _stream
        if self.current != self.n:
            raise RuntimeError(f"G has {self.current} of {self.n} columns")
        if slip.dtype != torch.float64 or not slip.is_cuda or slip.shape[0] != self.n or slip.dim() > 2:
            raise ValueError(f"slip must be a CUDA float64 tensor [{self.n}] or [{self.n}, k]")
        k = 1 if slip.dim() == 1 else slip.shape[1]
        S = slip.reshape(self.n, k).T.contiguous()  # [k][n]: one state per row
        G = self.G.contiguous()
        tb = self.t_boundary.contiguous()
        out = torch.empty(k, self.n, dtype=torch.float64, device=slip.device)
        _ffi.check(_ffi.lib().tdg_gf_traction_update(self.n, self.n, C.c_void_p(G.data_ptr()), self.n,
                                                     C.c_void_p(S.data_ptr()), self.n, k, C.c_void_p(tb.data_ptr()),
                                                     float(time), C.c_void_p(out.data_ptr()), self.n,
                                                     _stream(stream)))
        return out[0] if slip.dim() == 1 else out.T

    def save(self, path: str) -> None:
        save_checkpoint(path, self.G.cpu().numpy(), self.done, self.labels, self.fault.nbf)

    def load(self, path: str) -> int:
        """Loads a checkpoint (any facet order); returns the number of computed columns."""
        import torch
        G, done = load_checkpoint(path, self.labels, self.fault.nbf)
        self.G = torch.as_tensor(G, device="cuda")
        self.done = done
        return self.current
