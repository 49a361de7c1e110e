"""One operator across ranks: element partition, local meshes with a ghost layer, the ghost
exchange before every apply, and a distributed preconditioned CG.

tandem distributes a mesh by elements (ParMETIS), orders each rank's elements interior, copy,
ghost (src/form/DGOperatorTopo.h:27-40) and, in DGOperator::apply_ (src/form/DGOperator.h:384-393),
starts the ghost exchange, applies the interior elements, waits, and applies the rest.  Here:

* ``partition_elements``: recursive coordinate bisection of the element centroids (deterministic,
  parts differ by at most one element);
* ``local_mesh``: a rank's owned elements (ascending global id; they include tandem's "copy"
  elements) followed by one layer of ghost elements (the elements across the owned elements'
  interior facets).  Facets keep the global mesh's boundary codes and the global side order (side
  0 = the element with the smaller global id), so fault orientation and slip signs agree with the
  global operator.  The ghost layer's outer facets become artificial boundary facets with code
  None: their flux only reaches ghost rows, which the caller discards, so every owned row of the
  local operator equals the global operator's row (the facet penalty and the block-Jacobi blocks
  of owned elements see both sides of every facet).
* ``HaloPlan`` / ``HaloExchange``: per peer rank the owned elements it needs and the ghosts it
  owns, both in ascending global id, and the exchange of those element blocks with
  torch.distributed point-to-point messages (gloo with host tensors, nccl with device tensors).
* ``DistributedOperator`` / ``distributed_pcg``: y = A x on the owned rows with the exchange in
  front, dot products over owned rows (several per all-reduce), and PCG with an element-local
  preconditioner (block Jacobi of the owned elements) and two all-reduces per iteration -- the host
  restatement, run by the CPU tests with the oracle as each rank's operator;
* ``DeviceDistributedSolver``: the same solve on the device through the library
  (tdg_solve_distributed): the library's CG with its device-resident scalars, reliable updates and
  block-Jacobi kernels runs on the owned rows, and calls back for the ghost exchange before every
  apply and for the all-reduce of every dot product (nccl: device tensors on the solve's stream,
  nothing synchronises; gloo: staged through host memory).

The communication carries only ghost blocks (bs values per ghost element and right-hand side); the
apply itself is the single-mesh apply of the local operator.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import mesh as M


def _centroids(mesh: M.SimplexMesh) -> np.ndarray:
    return mesh.vertices[mesh.elements].mean(axis=1)


def partition_elements(mesh: M.SimplexMesh, nparts: int) -> np.ndarray:
    """part[e] in [0, nparts): recursive coordinate bisection of the element centroids along the
    widest extent, with the element counts split in proportion to the parts on each side."""
    if nparts < 1:
        raise ValueError("nparts must be positive")
    c = _centroids(mesh)
    part = np.zeros(mesh.num_elements, dtype=np.int32)

    def split(ids: np.ndarray, p0: int, n: int) -> None:
        if n == 1:
            part[ids] = p0
            return
        nl = n // 2
        ext = c[ids].max(axis=0) - c[ids].min(axis=0)
        axis = int(np.argmax(ext))
        order = ids[np.lexsort((ids, c[ids, axis]))]
        cut = (len(ids) * nl) // n
        split(order[:cut], p0, nl)
        split(order[cut:], p0 + nl, n - nl)

    split(np.arange(mesh.num_elements), 0, nparts)
    return part


def _neighbour_pairs(mesh: M.SimplexMesh) -> np.ndarray:
    up = mesh.facet_up
    inner = up[:, 0] != up[:, 1]
    return up[inner]


@dataclass
class HaloPlan:
    """Exchange lists of one rank: for each peer, local indices of the owned elements to send
    (send[q]) and of the ghost elements to receive (recv[q]), both in ascending global id."""
    send: dict = field(default_factory=dict)
    recv: dict = field(default_factory=dict)


@dataclass
class LocalMesh:
    mesh: M.SimplexMesh         # owned elements, then ghosts
    elements: np.ndarray        # global element id of each local element
    facets: np.ndarray          # global facet id of each local facet (slices facet data)
    n_owned: int
    plan: HaloPlan


def local_mesh(mesh: M.SimplexMesh, part: np.ndarray, rank: int) -> LocalMesh:
    """The rank's local mesh with one ghost layer (see the module docstring).  `mesh` must carry
    topology and geometry nodes."""
    part = np.asarray(part)
    owned = np.nonzero(part == rank)[0]
    pairs = _neighbour_pairs(mesh)
    is_owned = part == rank
    a, b = pairs[:, 0], pairs[:, 1]
    ghosts = np.unique(np.concatenate([b[is_owned[a] & ~is_owned[b]], a[is_owned[b] & ~is_owned[a]]]))
    elems = np.concatenate([owned, ghosts]).astype(np.int64)
    g2l = np.full(mesh.num_elements, -1, dtype=np.int64)
    g2l[elems] = np.arange(len(elems))

    # vertices renumbered monotonically, so every element's corners stay sorted
    gverts = np.unique(mesh.elements[elems])
    lm = M.SimplexMesh(mesh.dim, np.ascontiguousarray(mesh.vertices[gverts]),
                       np.searchsorted(gverts, mesh.elements[elems]).astype(np.int64))
    M.topology(lm, boundary_bc=M.BC_NONE)
    # side order of the global mesh: side 0 is the element with the smaller global id
    up, loc = lm.facet_up, lm.facet_local
    inner = up[:, 0] != up[:, 1]
    swap = inner & (elems[up[:, 0]] > elems[up[:, 1]])
    up[swap] = up[swap][:, ::-1]
    loc[swap] = loc[swap][:, ::-1]
    # boundary codes of the global facets (artificial boundary facets of the ghost layer: None)
    V = mesh.vertices.shape[0]
    if float(V) ** mesh.dim >= 2.0 ** 62:
        raise ValueError("too many vertices for the facet keys")
    gkey = np.ravel_multi_index(tuple(mesh.facets.T), (V,) * mesh.dim)
    order = np.argsort(gkey)
    lkey = np.ravel_multi_index(tuple(gverts[lm.facets].T), (V,) * mesh.dim)
    pos = np.searchsorted(gkey[order], lkey)
    found = (pos < len(gkey)) & (gkey[order][np.minimum(pos, len(gkey) - 1)] == lkey)
    if not np.all(found):
        raise ValueError("local facet missing from the global mesh")
    gf = order[pos]
    bc = mesh.facet_bc[gf].astype(np.int32)
    global_boundary = mesh.facet_up[gf, 0] == mesh.facet_up[gf, 1]
    local_boundary = ~inner
    bc[local_boundary & ~global_boundary] = M.BC_NONE
    lm.facet_bc = bc
    lm.geo_degree = mesh.geo_degree
    lm.geo_nodes = np.ascontiguousarray(mesh.geo_nodes[elems])
    if mesh.p2_nodes is not None:
        lm.p2_nodes = np.ascontiguousarray(mesh.p2_nodes[elems])
    lm.info = dict(rank=rank, n_owned=len(owned))

    # exchange lists
    plan = HaloPlan()
    peers = np.unique(part[ghosts]) if len(ghosts) else np.zeros(0, dtype=np.int32)
    for q in peers.tolist():
        recv = ghosts[part[ghosts] == q]
        plan.recv[q] = g2l[recv]
        own_a = is_owned[a] & (part[b] == q)
        own_b = is_owned[b] & (part[a] == q)
        send = np.unique(np.concatenate([a[own_a], b[own_b]]))
        plan.send[q] = g2l[send]
    return LocalMesh(lm, elems, gf.astype(np.int64), len(owned), plan)


class HaloExchange:
    """Fills the ghost blocks of a local vector (nrhs columns at stride ld, bs values per element)
    with the owning ranks' values.  Every rank of the group calls exchange() at the same point."""

    def __init__(self, plan: HaloPlan, bs: int, group=None):
        self.plan, self.bs, self.group = plan, bs, group
        self._idx = {}
        self._started = False

    def _entries(self, which: str, q: int, nrhs: int, ld: int, device):
        """Vector entries of the element list plan.<which>[q] over nrhs columns (cached)."""
        import torch
        key = (which, q, nrhs, ld, str(device))
        if key not in self._idx:
            e = torch.as_tensor(getattr(self.plan, which)[q], dtype=torch.int64, device=device)
            blk = (e[:, None] * self.bs + torch.arange(self.bs, device=device)[None, :]).reshape(-1)
            self._idx[key] = (blk[None, :] + ld * torch.arange(nrhs, device=device)[:, None]).reshape(-1)
        return self._idx[key]

    def exchange(self, x, nrhs: int = 1, ld: int | None = None) -> None:
        """The sends and receives go out as one batch (batch_isend_irecv: grouped under nccl, so
        two ranks that send to each other before receiving cannot block each other).  The first
        exchange starts with a barrier, since a rank without peers has nothing to batch and a
        group's first batch must include every rank."""
        import torch
        import torch.distributed as dist
        ld = x.numel() // nrhs if ld is None else ld
        ops, recvs = [], []
        for q in sorted(self.plan.send):
            buf = x.index_select(0, self._entries("send", q, nrhs, ld, x.device)).contiguous()
            ops.append(dist.P2POp(dist.isend, buf, q, self.group))
        for q in sorted(self.plan.recv):
            idx = self._entries("recv", q, nrhs, ld, x.device)
            buf = torch.empty(idx.numel(), dtype=x.dtype, device=x.device)
            ops.append(dist.P2POp(dist.irecv, buf, q, self.group))
            recvs.append((idx, buf))
        if not self._started:
            dist.barrier(group=self.group)
            self._started = True
        for r in (dist.batch_isend_irecv(ops) if ops else []):
            r.wait()
        for idx, buf in recvs:
            x.index_copy_(0, idx, buf)


class DistributedOperator:
    """y = A x on the owned rows of a local vector, with the ghost exchange in front.  apply_local
    computes the local operator on the whole local vector (any device or host implementation with
    the signature apply_local(x, y, nrhs, ld)); dot() reduces over owned rows of all ranks."""

    def __init__(self, lmesh: LocalMesh, bs: int, apply_local, group=None):
        self.lm, self.bs, self.apply_local, self.group = lmesh, bs, apply_local, group
        self.halo = HaloExchange(lmesh.plan, bs, group)
        self.n_local = len(lmesh.elements) * bs
        self.n_owned = lmesh.n_owned * bs

    def apply(self, x, y) -> None:
        self.halo.exchange(x)
        self.apply_local(x, y)
        y[self.n_owned:] = 0

    def dot(self, a, b) -> float:
        return self.dots((a, b))[0]

    def dots(self, *pairs) -> list[float]:
        """Several dot products over the owned rows of all ranks with one all-reduce."""
        import torch
        import torch.distributed as dist
        n = self.n_owned
        s = torch.stack([torch.dot(a[:n], b[:n]).to(torch.float64) for a, b in pairs])
        dist.all_reduce(s, group=self.group)
        return [float(v) for v in s.tolist()]


def distributed_pcg(A: DistributedOperator, precondition, b, x, rtol: float = 1e-10,
                    max_iterations: int = 10000) -> dict:
    """Preconditioned CG over the ranks: b, x local vectors (owned rows meaningful, x's ghost rows
    overwritten by the exchange), precondition(r, z) element-local (it must write z's owned rows).
    The stopping test ||r|| <= rtol ||b|| uses the recurrence residual, as PETSc's KSPCG does."""
    import torch
    r = torch.zeros_like(b)
    q = torch.zeros_like(b)
    A.apply(x, q)
    r[:A.n_owned] = b[:A.n_owned] - q[:A.n_owned]
    z = torch.zeros_like(b)
    precondition(r, z)
    p = z.clone()
    rz, bb, rr = A.dots((r, z), (b, b), (r, r))
    bn, rn = bb ** 0.5, rr ** 0.5
    it = 0
    while it < max_iterations and rn > rtol * bn:
        A.apply(p, q)
        alpha = rz / A.dot(p, q)
        x[:A.n_owned] += alpha * p[:A.n_owned]
        r[:A.n_owned] -= alpha * q[:A.n_owned]
        precondition(r, z)
        rz1, rr = A.dots((r, z), (r, r))  # two all-reduces per iteration in all
        p[:A.n_owned] = z[:A.n_owned] + (rz1 / rz) * p[:A.n_owned]
        rz = rz1
        rn = rr ** 0.5
        it += 1
    return dict(iterations=it, rel_residual=rn / bn if bn > 0 else 0.0, converged=rn <= rtol * bn)


def device_operator(lmesh: LocalMesh, degree: int, kind: int, quad, c0_Q, c1_Q=None, precision: int = 0,
                    group=None):
    """A rank's local operator on its GPU with the ghost exchange in front (use the nccl backend,
    one process per GPU): returns (the local DGOperator, the DistributedOperator, a block-Jacobi
    precondition(r, z)).  c0_Q / c1_Q are the global material arrays [E, Nq]; precision selects the
    apply arithmetic (FP64 or MIXED with FP64 vectors).  Vectors are local device float64 tensors
    of len(lmesh.elements) * bs entries, owned blocks first."""
    from .operator import FP64, DGOperator
    op = DGOperator(lmesh.mesh, degree, kind, quad)
    op.set_material(np.ascontiguousarray(c0_Q[lmesh.elements]),
                    None if c1_Q is None else np.ascontiguousarray(c1_Q[lmesh.elements]))
    op.bjacobi_setup(FP64)
    A = DistributedOperator(lmesh, op.bs, lambda x, y: op.apply(x, y, precision), group)
    return op, A, (lambda r, z: op.bjacobi_apply(r, z))


class _DeviceBuffer:
    """A device array seen by torch without a copy (CUDA array interface)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None}


class DeviceDistributedSolver:
    """One rank's part of a CG solve over a distributed operator on the device (tdg_solve_distributed).

    op: the rank's local DGOperator (lmesh's mesh: owned elements, then the ghost layer), with the
    block-Jacobi preconditioner set up; vectors are local device float64 tensors of op.ndof entries,
    owned blocks first.  The library calls back before every apply (the ghost exchange of HaloExchange)
    and for every dot product (all-reduce over the group).  With the nccl backend the callbacks enqueue
    the collectives on the solve's stream; with gloo they stage through host memory."""

    def __init__(self, op, lmesh: LocalMesh, group=None):
        import torch.distributed as dist
        from . import _ffi
        self.op, self.lm, self.group = op, lmesh, group
        self.halo = HaloExchange(lmesh.plan, op.bs, group)
        self.host = dist.get_backend(group) != "nccl"
        self.errors: list[str] = []
        self._exchange_cb = _ffi.EXCHANGE_FN(self._exchange)
        self._allreduce_cb = _ffi.ALLREDUCE_FN(self._allreduce)

    @staticmethod
    def _stream(ptr):
        import torch
        return torch.cuda.ExternalStream(ptr) if ptr else torch.cuda.default_stream()

    def _exchange(self, ctx, v, stream) -> int:
        import torch
        try:
            t = torch.as_tensor(_DeviceBuffer(v, self.op.ndof), device="cuda")
            with torch.cuda.stream(self._stream(stream)):
                if self.host:
                    h = t.cpu()  # synchronises the stream
                    self.halo.exchange(h)
                    t.copy_(h)
                else:
                    self.halo.exchange(t)
            return 0
        except Exception as e:  # noqa: BLE001 - reported to the library as a failed callback
            self.errors.append(repr(e))
            return 1

    def _allreduce(self, ctx, values, count, stream) -> int:
        import torch
        import torch.distributed as dist
        try:
            t = torch.as_tensor(_DeviceBuffer(values, count), device="cuda")
            with torch.cuda.stream(self._stream(stream)):
                if self.host:
                    h = t.cpu()
                    dist.all_reduce(h, group=self.group)
                    t.copy_(h)
                else:
                    dist.all_reduce(t, group=self.group)
            return 0
        except Exception as e:  # noqa: BLE001
            self.errors.append(repr(e))
            return 1

    def solve(self, b, x, precision: int = 0, rtol: float = 1e-10, max_iterations: int = 20000, stream=None,
              check: bool = True) -> dict:
        """Solves A x = b over the ranks (b, x: local device vectors, owned rows meaningful; x holds
        the initial guess).  Every rank of the group calls it with the same arguments."""
        import ctypes as C
        from . import _ffi
        from .operator import _check_vec, _stream
        _check_vec(b, 0, self.op.ndof)
        _check_vec(x, 0, self.op.ndof)
        opts = _ffi.SolveOpts(precision, max_iterations, rtol, 0.0, 0, 0, _ffi.TDG_KSP_CG, 0)
        st = _ffi.SolveStats()
        rc = _ffi.lib().tdg_solve_distributed(self.op._h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()),
                                              self.lm.n_owned, C.byref(opts), C.byref(st), self._exchange_cb,
                                              self._allreduce_cb, None, _stream(stream))
        stats = dict(iterations=st.iterations, outer=st.outer, rel_residual=st.rel_residual, seconds=st.seconds,
                     converged=bool(st.converged))
        if rc != 0 and (check or rc != _ffi.ERRORS_BY_NAME["TDG_E_DIVERGED"]):
            raise _ffi.TdgError(f"{_ffi.ERRORS.get(rc, rc)}: {_ffi.lib().tdg_last_error().decode()} {stats} "
                                f"{self.errors}")
        return stats
