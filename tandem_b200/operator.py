"""Host-side mirror of tandem's DG operator interface over the C ABI.

``DGOperator`` plays the role of tandem's ``AbstractDGOperator`` / ``DGOperator<LOP>``
(src/form/AbstractDGOperator.h:18-52): ``block_size``, ``num_local_elements``, ``apply``, ``rhs``,
the block-Jacobi part of ``assemble``, ``flops_apply``; ``solve`` plays ``PetscLinearSolver``
(app/common/PetscLinearSolver.cpp) with CG + block Jacobi on the device.  Vectors are torch CUDA
tensors in tandem's block layout (x[e * bs + k + Nbf * p]); every compute call goes to the native
library, there is no host fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _ffi
from .mesh import SimplexMesh

POISSON, ELASTICITY = _ffi.TDG_POISSON, _ffi.TDG_ELASTICITY
FP64, FP32, MIXED, TF32 = _ffi.TDG_FP64, _ffi.TDG_FP32, _ffi.TDG_MIXED, _ffi.TDG_TF32
FAMILIES = ("tensor", "simt", "face", "face2", "tc05")
MG_STRATEGIES = ("twolevel", "logarithmic", "full")  # MGStrategy (app/common/MGConfig.h:8)
PRECONDITIONERS = ("bjacobi", "mg")
MG_COARSE_SPACES = ("dg", "p1")
KSP_METHODS = ("cg", "fgmres")  # TDG_KSP_CG, TDG_KSP_FGMRES


def _c(a: np.ndarray, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


def _stream(stream) -> C.c_void_p:
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(getattr(stream, "cuda_stream", stream))


@dataclass
class Quadrature:
    """Volume and facet rules on the unit simplex (tandem's volRule / fctRule)."""
    vol_x: np.ndarray
    vol_w: np.ndarray
    fct_x: np.ndarray
    fct_w: np.ndarray

    @staticmethod
    def conical(dim: int, order: int) -> "Quadrature":
        from .refelem import conical_rule
        vx, vw = conical_rule(dim, order)
        fx, fw = conical_rule(dim - 1, order)
        return Quadrature(vx, vw, fx, fw)


class DGOperator:
    def __init__(self, mesh: SimplexMesh, degree: int, kind: int, quad: Quadrature):
        self.mesh, self.degree, self.kind, self.quad = mesh, degree, kind, quad
        L = _ffi.lib()
        D = mesh.dim
        self._keep = dict(
            geo=_c(mesh.geo_nodes, np.float64), up=_c(mesh.facet_up, np.int64),
            loc=_c(mesh.facet_local, np.int32), bc=_c(mesh.facet_bc, np.int32),
            vx=_c(quad.vol_x, np.float64), vw=_c(quad.vol_w, np.float64),
            fx=_c(quad.fct_x, np.float64), fw=_c(quad.fct_w, np.float64))
        k = self._keep
        desc = _ffi.MeshDesc(D, degree, mesh.geo_degree, 0, mesh.num_elements, mesh.num_facets,
                             k["geo"].ctypes.data, k["up"].ctypes.data, k["loc"].ctypes.data,
                             k["bc"].ctypes.data)
        qd = _ffi.Quadrature(len(k["vw"]), len(k["fw"]), k["vx"].ctypes.data, k["vw"].ctypes.data,
                             k["fx"].ctypes.data, k["fw"].ctypes.data)
        h = C.c_void_p()
        _ffi.check(L.tdg_create(C.byref(desc), C.byref(qd), kind, C.byref(h)))
        self._h = h
        sizes = (C.c_int64 * 8)()
        _ffi.check(L.tdg_sizes(h, sizes))
        self.bs, self.nbf, self.Q, self.Nq, self.nq, self.E, self.F, self.dim = [int(s) for s in sizes]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _ffi.lib().tdg_destroy(h)
            except Exception:  # noqa: BLE001 - interpreter shutdown: the library may be gone
                pass
            self._h = None

    # -- sizes (AbstractDGOperator) --------------------------------------------------------------
    def block_size(self) -> int:
        return self.bs

    def num_local_elements(self) -> int:
        return self.E

    @property
    def ndof(self) -> int:
        return self.E * self.bs

    # -- geometry for the caller's functionals -------------------------------------------------
    def volume_coords(self) -> np.ndarray:
        out = np.zeros((self.E, self.Nq, self.dim))
        _ffi.check(_ffi.lib().tdg_volume_coords(self._h, out.ctypes.data))
        return out

    def facet_coords(self) -> np.ndarray:
        out = np.zeros((self.F, self.nq, self.dim))
        _ffi.check(_ffi.lib().tdg_facet_coords(self._h, out.ctypes.data))
        return out

    def facet_normals(self) -> np.ndarray:
        out = np.zeros((self.F, self.nq, self.dim))
        _ffi.check(_ffi.lib().tdg_facet_normals(self._h, out.ctypes.data))
        return out

    # -- material --------------------------------------------------------------------------------
    def set_material(self, c0_Q: np.ndarray, c1_Q: np.ndarray | None = None) -> None:
        a = _c(c0_Q, np.float64).reshape(self.E, self.Nq)
        b = None if c1_Q is None else _c(c1_Q, np.float64).reshape(self.E, self.Nq)
        self._mat = (a, b)
        _ffi.check(_ffi.lib().tdg_set_material(self._h, a.ctypes.data, None if b is None else b.ctypes.data))

    def update_material(self, c0_Q: np.ndarray, c1_Q: np.ndarray | None = None) -> None:
        """Replaces the material but keeps the preconditioner set up for the previous one
        (tdg_update_material): for nearby materials (finite differences, line searches)."""
        a = _c(c0_Q, np.float64).reshape(self.E, self.Nq)
        b = None if c1_Q is None else _c(c1_Q, np.float64).reshape(self.E, self.Nq)
        self._mat = (a, b)
        _ffi.check(_ffi.lib().tdg_update_material(self._h, a.ctypes.data, None if b is None else b.ctypes.data))

    def material_nodal(self, c: int) -> np.ndarray:
        out = np.zeros((self.E, self.nbf))
        _ffi.check(_ffi.lib().tdg_material_nodal(self._h, c, out.ctypes.data))
        return out

    def penalty(self) -> np.ndarray:
        out = np.zeros(self.F)
        _ffi.check(_ffi.lib().tdg_penalty(self._h, out.ctypes.data))
        return out

    # -- hot path --------------------------------------------------------------------------------
    def apply(self, x, y, precision: int = FP64, nrhs: int = 1, ld: int | None = None, stream=None) -> None:
        """y = A x on the device (PetscDGShell::apply)."""
        ld = self.ndof if ld is None else ld
        _check_vec(x, precision, nrhs * ld)
        _check_vec(y, precision, nrhs * ld)
        _ffi.check(_ffi.lib().tdg_apply(self._h, precision, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                        nrhs, ld, _stream(stream)))

    def apply_host(self, x, y, precision: int = FP64, count: int = 1, stride: int | None = None,
                   stream=None) -> None:
        """y_i = A x_i for `count` vectors in host memory (CPU tensors, pinned for overlap) at
        `stride` entries apart (default ndof; 0 = the same vector every time): copy in, apply and
        copy out, the copies of neighbouring vectors overlapping the apply (tdg_apply_host).
        Ordered on `stream` like a device apply."""
        import torch
        stride = self.ndof if stride is None else stride
        want = torch.float32 if precision == FP32 else torch.float64
        need = self.ndof + (count - 1) * stride
        for t in (x, y):
            if t.is_cuda or t.dtype != want or not t.is_contiguous() or t.numel() < need:
                raise ValueError(f"expected a contiguous host {want} tensor with >= {need} entries")
        _ffi.check(_ffi.lib().tdg_apply_host(self._h, precision, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                             count, stride, _stream(stream)))

    # -- explicit wave operator (Elasticity::wave_rhs) ------------------------------------------
    def set_density(self, rho_Q: np.ndarray) -> None:
        """Density at the volume points [E, Nq] (elasticity; default 1)."""
        r = _c(rho_Q, np.float64).reshape(self.E, self.Nq)
        self._rho = r
        _ffi.check(_ffi.lib().tdg_set_density(self._h, r.ctypes.data))

    def apply_inverse_mass(self, x, y, nrhs: int = 1, ld: int | None = None, stream=None) -> None:
        """y = -(1/rho)-weighted inverse mass of x (tandem's apply_inverse_mass)."""
        ld = self.ndof if ld is None else ld
        _check_vec(x, FP64, nrhs * ld)
        _check_vec(y, FP64, nrhs * ld)
        _ffi.check(_ffi.lib().tdg_apply_inverse_mass(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                                     nrhs, ld, _stream(stream)))

    def wave_rhs(self, x, y, b=None, nrhs: int = 1, ld: int | None = None, stream=None) -> None:
        """y = inverse mass of (A x - b), the acceleration of rho u'' = b - A u; b: boundary-data
        right-hand side (device FP64) or None."""
        ld = self.ndof if ld is None else ld
        _check_vec(x, FP64, nrhs * ld)
        _check_vec(y, FP64, nrhs * ld)
        bp = None
        if b is not None:
            _check_vec(b, FP64, nrhs * ld)
            bp = C.c_void_p(b.data_ptr())
        _ffi.check(_ffi.lib().tdg_wave_rhs(self._h, C.c_void_p(x.data_ptr()), bp, C.c_void_p(y.data_ptr()), nrhs,
                                           ld, _stream(stream)))

    def autotune(self, precision: int = FP64, nrhs: int = 1, stream=None) -> list[dict]:
        """Times the candidate apply launch configurations on this operator and keeps the fastest
        for later applies and solves in `precision` (tdg_autotune).  Returns every measurement."""
        entries = (_ffi.TuneEntry * 64)()
        n = C.c_int(0)
        _ffi.check(_ffi.lib().tdg_autotune(self._h, precision, nrhs, _stream(stream), entries, 64, C.byref(n)))
        return [dict(family=FAMILIES[e.family], ctas_per_sm=e.ctas_per_sm, tile=e.tile, ms=e.ms)
                for e in entries[:n.value]]

    def set_apply_config(self, precision: int, family: str, ctas_per_sm: int = 0, tile: int = 0) -> None:
        """Selects the apply kernel explicitly: family "tensor" (element-centric tensor cores),
        "face" (face-centric), "face2" (face-centric, software-pipelined; FP64), "tc05" (FP32:
        face-centric with the volume term on tcgen05) or "simt";
        ctas_per_sm 0 = the default occupancy; tile (FP64 "face2" only) = volume points per pass of
        its volume kernel, a multiple of 8 (3D) or 4 (2D), 0 = automatic (tdg_set_apply_tile)."""
        _ffi.check(_ffi.lib().tdg_set_apply_config(self._h, precision, FAMILIES.index(family), ctas_per_sm))
        _ffi.check(_ffi.lib().tdg_set_apply_tile(self._h, precision, tile))

    def flops_apply(self) -> int:
        return int(_ffi.lib().tdg_flops_apply(self._h))

    def bytes_apply(self, precision: int = FP64) -> int:
        return int(_ffi.lib().tdg_bytes_apply(self._h, precision))

    def bjacobi_setup(self, precision: int = FP64, stream=None) -> None:
        _ffi.check(_ffi.lib().tdg_bjacobi_setup(self._h, precision, _stream(stream)))

    def bjacobi_apply(self, r, z, precision: int = FP64, nrhs: int = 1, ld: int | None = None, stream=None) -> None:
        ld = self.ndof if ld is None else ld
        _check_vec(r, precision, nrhs * ld)
        _check_vec(z, precision, nrhs * ld)
        _ffi.check(_ffi.lib().tdg_bjacobi_apply(self._h, precision, C.c_void_p(r.data_ptr()),
                                                C.c_void_p(z.data_ptr()), nrhs, ld, _stream(stream)))

    def bjacobi_blocks(self) -> np.ndarray:
        out = np.zeros((self.E, self.bs, self.bs))
        _ffi.check(_ffi.lib().tdg_bjacobi_blocks(self._h, out.ctypes.data))
        # stored column-major per block: out[e, col, row] -> transpose to [e, row, col]
        return np.ascontiguousarray(out.transpose(0, 2, 1))

    # -- p-multigrid preconditioner (PetscLinearSolver::setup_mg + mg_cheby.cfg) -------------------
    def mg_setup(self, strategy: str = "logarithmic", coarse_degree: int = 1, smooth_its: int = 10,
                 esteig: tuple[float, float] = (0.01, 1.1), esteig_steps: int = 10, coarse_rtol: float = 0.1,
                 coarse_max_it: int = 1000, smooth_precision: int = FP64, coarse_space: str = "p1",
                 stream=None) -> None:
        """Builds the p-multigrid hierarchy (tdg_mg_setup): levels by MGConfig strategy, Galerkin
        coarse operators, Chebyshev smoothers on esteig x lambda_max(D^-1 A) with point Jacobi, and
        a block-Jacobi CG coarse solve -- on the coarsest DG level (coarse_space "dg") or on the
        continuous P1 space below it ("p1").  smooth_precision MIXED runs the finest level's
        smoother applies in FP32 arithmetic and the smoothed levels below it on FP32 copies of
        their blocks (FP64 vectors and accumulation); TF32 runs those smoother applies in one TF32
        tensor-core pass instead of three."""
        o = _ffi.MgOpts(MG_STRATEGIES.index(strategy), coarse_degree, smooth_its, esteig[0], esteig[1],
                        esteig_steps, coarse_rtol, coarse_max_it, smooth_precision,
                        MG_COARSE_SPACES.index(coarse_space))
        _ffi.check(_ffi.lib().tdg_mg_setup(self._h, C.byref(o), _stream(stream)))

    def mg_apply(self, r, z, nrhs: int = 1, ld: int | None = None, stream=None) -> None:
        """z = M r, one multigrid V-cycle per right-hand side (FP64 device vectors)."""
        ld = self.ndof if ld is None else ld
        _check_vec(r, FP64, nrhs * ld)
        _check_vec(z, FP64, nrhs * ld)
        _ffi.check(_ffi.lib().tdg_mg_apply(self._h, C.c_void_p(r.data_ptr()), C.c_void_p(z.data_ptr()), nrhs, ld,
                                           _stream(stream)))

    def set_preconditioner(self, pc: str) -> None:
        """Preconditioner of the solves: "bjacobi" (default) or "mg" (flexible CG around the V-cycle)."""
        _ffi.check(_ffi.lib().tdg_set_preconditioner(self._h, PRECONDITIONERS.index(pc)))

    def mg_info(self) -> dict:
        n = C.c_int(0)
        deg, bs = (C.c_int * 8)(), (C.c_int * 8)()
        lmax = (C.c_double * 8)()
        its = C.c_int64(0)
        _ffi.check(_ffi.lib().tdg_mg_info(self._h, C.byref(n), 8, deg, bs, lmax, C.byref(its)))
        k = n.value
        return dict(levels=k, degrees=list(deg[:k]), block_sizes=list(bs[:k]), lambda_max=list(lmax[:k]),
                    coarse_iterations=its.value)

    # -- projection and evaluation (AbstractDGOperator::project / solution; host) ---------------
    def project(self, U_Q: np.ndarray) -> np.ndarray:
        """Coefficients [ndof] of values at the volume points U_Q [E, Q, Nq] (Elasticity::project:
        weight-adjusted inverse mass of the L2 right-hand side)."""
        u = _c(U_Q, np.float64).reshape(self.E, self.Q, self.Nq)
        y = np.zeros(self.ndof)
        _ffi.check(_ffi.lib().tdg_project(self._h, u.ctypes.data, y.ctypes.data))
        return y

    def evaluate(self, x, points: np.ndarray) -> np.ndarray:
        """The discrete function x at unit-simplex points [np, dim] of every element: [E, Q, np]."""
        pts = _c(points, np.float64).reshape(-1, self.dim)
        xs = self._host_solution(x)
        out = np.zeros((self.E, self.Q, pts.shape[0]))
        _ffi.check(_ffi.lib().tdg_evaluate(self._h, xs.ctypes.data, pts.shape[0], pts.ctypes.data, out.ctypes.data))
        return out

    # -- error norms (Error<D>::L2 / H1_semi; host post-processing) ------------------------------
    def rule_coords(self, points: np.ndarray) -> np.ndarray:
        """Physical coordinates [E, np, dim] of unit-simplex points [np, dim] on every element."""
        pts = _c(points, np.float64).reshape(-1, self.dim)
        out = np.zeros((self.E, pts.shape[0], self.dim))
        _ffi.check(_ffi.lib().tdg_rule_coords(self._h, pts.shape[0], pts.ctypes.data, out.ctypes.data))
        return out

    @staticmethod
    def _host_solution(x) -> np.ndarray:
        if hasattr(x, "detach"):
            x = x.detach().cpu().numpy()
        return _c(x, np.float64)

    def error_l2(self, x, points: np.ndarray, weights: np.ndarray, ref: np.ndarray) -> float:
        """||x - ref||_L2 with the given rule; ref [E, Q, np] at rule_coords(points) (tandem's
        Error::L2 uses simplexQuadratureRule(20), e.g. conical_rule(dim, 20))."""
        pts = _c(points, np.float64).reshape(-1, self.dim)
        w = _c(weights, np.float64)
        r = _c(ref, np.float64).reshape(self.E, self.Q, pts.shape[0])
        xs = self._host_solution(x)
        out = C.c_double(0.0)
        _ffi.check(_ffi.lib().tdg_error_l2(self._h, xs.ctypes.data, pts.shape[0], pts.ctypes.data, w.ctypes.data,
                                           r.ctypes.data, C.byref(out)))
        return out.value

    def error_h1_semi(self, x, points: np.ndarray, weights: np.ndarray, refgrad: np.ndarray) -> float:
        """|x - ref|_H1 (gradient L2 norm) with the given rule; refgrad [E, Q, dim, np]."""
        pts = _c(points, np.float64).reshape(-1, self.dim)
        w = _c(weights, np.float64)
        r = _c(refgrad, np.float64).reshape(self.E, self.Q, self.dim, pts.shape[0])
        xs = self._host_solution(x)
        out = C.c_double(0.0)
        _ffi.check(_ffi.lib().tdg_error_h1_semi(self._h, xs.ctypes.data, pts.shape[0], pts.ctypes.data,
                                                w.ctypes.data, r.ctypes.data, C.byref(out)))
        return out.value

    def mg_colouring(self) -> tuple[np.ndarray, int]:
        """Distance-2 element colouring of the Galerkin probing (host only): colour [E], count."""
        out = np.zeros(self.E, dtype=np.int32)
        n = C.c_int(0)
        _ffi.check(_ffi.lib().tdg_mg_colouring(self._h, out.ctypes.data, C.byref(n)))
        return out, n.value

    def mg_vertex_numbering(self) -> tuple[np.ndarray, int]:
        """Vertices of the continuous P1 coarse space (host only): vid [E, dim + 1], count."""
        out = np.zeros((self.E, self.dim + 1), dtype=np.int32)
        n = C.c_int64(0)
        _ffi.check(_ffi.lib().tdg_mg_vertex_numbering(self._h, out.ctypes.data, C.byref(n)))
        return out, n.value

    def mg_level_matrix(self, level: int) -> tuple[np.ndarray, np.ndarray]:
        """Galerkin operator of a coarse level: blocks [E, NB, bs, bs] (row, column) and the
        neighbour table [E, NB] (slot 0 the element, 1 + f across face f, -1 none)."""
        info = self.mg_info()
        bs = info["block_sizes"][level]
        NB = self.dim + 2
        blocks = np.zeros((self.E, NB, bs, bs))
        nbr = np.zeros((self.E, NB), dtype=np.int32)
        _ffi.check(_ffi.lib().tdg_mg_level_matrix(self._h, level, blocks.ctypes.data, nbr.ctypes.data))
        return np.ascontiguousarray(blocks.transpose(0, 1, 3, 2)), nbr

    def rhs(self, force_Q: np.ndarray | None = None, bc_q: np.ndarray | None = None) -> np.ndarray:
        """Right-hand side (DGOperator::rhs): force_Q [E, Q, Nq], bc_q [F, Q, nq]."""
        b = np.zeros(self.ndof)
        f = None if force_Q is None else _c(force_Q, np.float64).reshape(self.E, self.Q, self.Nq)
        g = None if bc_q is None else _c(bc_q, np.float64).reshape(self.F, self.Q, self.nq)
        _ffi.check(_ffi.lib().tdg_rhs(self._h, None if f is None else f.ctypes.data,
                                      None if g is None else g.ctypes.data, b.ctypes.data))
        return b

    def solve(self, b, x, precision: int = FP64, rtol: float = 1e-10, max_iterations: int = 20000,
              inner_rtol: float = 0.0, max_outer: int = 0, use_graphs: bool = True, nrhs: int = 1,
              ld: int | None = None, stream=None, check: bool = True, method: str = "cg",
              restart: int = 30) -> dict:
        """Preconditioned CG on the device: FP64; MIXED (FP64 recurrence around the FP32
        tensor-core operator and FP32 block inverses or FP32 fine-level multigrid smoothing); or
        FP32 (operator, preconditioner and recurrence in FP32; block Jacobi only).  The
        preconditioner is block Jacobi or, after set_preconditioner("mg"), the multigrid V-cycle
        (flexible CG).  The solution and the true residual are FP64 in every mode (reliable
        updates).  inner_rtol: reliable-update threshold (0 = default).  method "fgmres": restarted
        flexible GMRES(restart) (FP64 or MIXED; iterations = Arnoldi steps, outer = cycles).  Raises
        on non-convergence unless check=False (then the stats report it)."""
        ld = self.ndof if ld is None else ld
        _check_vec(b, FP64, nrhs * ld)
        _check_vec(x, FP64, nrhs * ld)
        opts = _ffi.SolveOpts(precision, max_iterations, rtol, inner_rtol, max_outer, int(use_graphs),
                              KSP_METHODS.index(method), restart)
        st = _ffi.SolveStats()
        rc = _ffi.lib().tdg_solve(self._h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), nrhs, ld,
                                  C.byref(opts), C.byref(st), _stream(stream))
        stats = dict(iterations=st.iterations, outer=st.outer, rel_residual=st.rel_residual,
                     seconds=st.seconds, converged=bool(st.converged), fp64_iterations=st.fp64_iterations)
        if rc != 0 and (check or rc != _ffi.ERRORS_BY_NAME["TDG_E_DIVERGED"] or not np.isfinite(st.rel_residual)):
            raise _ffi.TdgError(f"{_ffi.ERRORS.get(rc, rc)}: {_ffi.lib().tdg_last_error().decode()} {stats}")
        return stats


def solve_segmented(op: DGOperator, b, x, elem_offsets, precision: int = FP64, rtol: float = 1e-10,
                    max_iterations: int = 20000, inner_rtol: float = 0.0, max_outer: int = 0,
                    use_graphs: bool = True, stream=None, check: bool = True, method: str = "cg",
                    restart: int = 30):
    """Independent problems held in one block-diagonal operator (a mesh union): one apply and one
    preconditioner launch per iteration cover every problem, each problem has its own CG scalars
    and stopping test.  Returns (aggregate stats, per-problem relative residuals); with
    check=False an iteration limit or stall is reported in the stats instead of raised."""
    off = np.ascontiguousarray(elem_offsets, dtype=np.int64)
    nseg = len(off) - 1
    _check_vec(b, FP64, op.ndof)
    _check_vec(x, FP64, op.ndof)
    opts = _ffi.SolveOpts(precision, max_iterations, rtol, inner_rtol, max_outer, int(use_graphs),
                          KSP_METHODS.index(method), restart)
    st = _ffi.SolveStats()
    rel = np.zeros(nseg)
    rc = _ffi.lib().tdg_solve_segmented(op._h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), nseg,
                                        off.ctypes.data, C.byref(opts), C.byref(st), rel.ctypes.data, _stream(stream))
    stats = dict(iterations=st.iterations, outer=st.outer, rel_residual=st.rel_residual, seconds=st.seconds,
                 converged=bool(st.converged), fp64_iterations=st.fp64_iterations)
    if rc != 0 and (check or rc != _ffi.ERRORS_BY_NAME["TDG_E_DIVERGED"] or not np.isfinite(st.rel_residual)):
        raise _ffi.TdgError(f"{_ffi.ERRORS.get(rc, rc)}: {_ffi.lib().tdg_last_error().decode()} {stats}")
    return stats, rel


def _check_vec(t, precision: int, n: int) -> None:
    import torch
    want = torch.float32 if precision == FP32 else torch.float64
    if not (t.is_cuda and t.dtype == want and t.is_contiguous() and t.numel() >= n):
        raise ValueError(f"expected a contiguous CUDA {want} tensor with >= {n} entries, got "
                         f"{t.dtype} device={t.device} numel={t.numel()}")


class Fault:
    """Fault coupling of a Poisson operator (tandem's Adapter<Poisson> over the fault facets):
    slip -> right-hand side and displacement -> on-fault traction, batched over right-hand sides."""

    def __init__(self, op: DGOperator, facets: np.ndarray, ref_normal):
        self.op = op
        self._facets = np.ascontiguousarray(facets, dtype=np.int64)
        self._ref = np.ascontiguousarray(ref_normal, dtype=np.float64)
        h = C.c_void_p()
        _ffi.check(_ffi.lib().tdg_fault_create(op._h, len(self._facets), self._facets.ctypes.data,
                                               self._ref.ctypes.data, C.byref(h)))
        self._h = h
        sizes = (C.c_int64 * 2)()
        _ffi.check(_ffi.lib().tdg_fault_sizes(h, sizes))
        self.nfault, self.nbf = int(sizes[0]), int(sizes[1])
        self.ncoef = self.nfault * self.nbf

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _ffi.lib().tdg_fault_destroy(h)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
            self._h = None

    def slip_rhs(self, slip, b, nrhs: int = 1, stream=None) -> None:
        """b += rhs of slip; slip [nrhs, ncoef], b [nrhs, ndof] (CUDA float64)."""
        _check_vec(slip, FP64, nrhs * self.ncoef)
        _check_vec(b, FP64, nrhs * self.op.ndof)
        _ffi.check(_ffi.lib().tdg_fault_slip_rhs(self._h, C.c_void_p(slip.data_ptr()), self.ncoef,
                                                 C.c_void_p(b.data_ptr()), nrhs, self.op.ndof, _stream(stream)))

    def traction(self, u, slip, out, nrhs: int = 1, stream=None) -> None:
        """out[nrhs, ncoef] = traction of displacement u [nrhs, ndof] and slip [nrhs, ncoef]."""
        _check_vec(u, FP64, nrhs * self.op.ndof)
        _check_vec(out, FP64, nrhs * self.ncoef)
        sp = None if slip is None else C.c_void_p(slip.data_ptr())
        _ffi.check(_ffi.lib().tdg_fault_traction(self._h, C.c_void_p(u.data_ptr()), self.op.ndof, sp, self.ncoef,
                                                 C.c_void_p(out.data_ptr()), self.ncoef, nrhs, _stream(stream)))


def greens_function(op: DGOperator, fault: Fault, precision: int = FP64, rtol: float = 1e-10,
                    columns=None, batch: int | None = None, **solve_kw):
    """Discrete Green's function G[:, i] = traction(solve(rhs(slip = e_i))) for the fault basis
    coefficients `columns` (all by default), solved as batched multi-right-hand-side launches
    (tandem: one KSPSolve per column, app/form/SeasQDDiscreteGreenOperator.cpp:519-574).
    Returns (G [ncoef, ncols] as a CUDA tensor, list of per-batch solve statistics)."""
    import torch
    cols = np.arange(fault.ncoef) if columns is None else np.asarray(columns)
    batch = len(cols) if batch is None else batch
    G = torch.zeros(fault.ncoef, len(cols), dtype=torch.float64, device="cuda")
    stats = []
    for s in range(0, len(cols), batch):
        c = cols[s:s + batch]
        n = len(c)
        slip = torch.zeros(n, fault.ncoef, dtype=torch.float64, device="cuda")
        slip[torch.arange(n, device="cuda"), torch.as_tensor(c, device="cuda")] = 1.0
        b = torch.zeros(n, op.ndof, dtype=torch.float64, device="cuda")
        fault.slip_rhs(slip, b, n)
        x = torch.zeros_like(b)
        st = op.solve(b, x, precision=precision, rtol=rtol, nrhs=n, **solve_kw)
        stats.append(st)
        T = torch.empty(n, fault.ncoef, dtype=torch.float64, device="cuda")
        fault.traction(x, slip, T, n)
        G[:, s:s + n] = T.T
    return G, stats


def mg_level_degrees(strategy: str, coarse_degree: int, degree: int) -> list[int]:
    """Level degrees, coarsest first (MGConfig::levels)."""
    out = (C.c_int * 16)()
    n = _ffi.lib().tdg_mg_level_degrees(MG_STRATEGIES.index(strategy), coarse_degree, degree, out)
    if n < 0:
        _ffi.check(n)
    return list(out[:n])


def mg_interpolation(dim: int, kind: int, n_to: int, n_from: int) -> np.ndarray:
    """Reference interpolation matrix of one component, [Nbf(n_to), Nbf(n_from)]."""
    from math import comb
    out = np.zeros((comb(n_to + dim, dim), comb(n_from + dim, dim)))
    _ffi.check(_ffi.lib().tdg_mg_interpolation(dim, kind, n_to, n_from, out.ctypes.data))
    return out


def mg_p1_embedding(dim: int, kind: int, degree: int) -> np.ndarray:
    """Coefficients [Nbf(degree), dim + 1] of each corner's hat function in the operator's space."""
    from math import comb
    out = np.zeros((comb(degree + dim, dim), dim + 1))
    _ffi.check(_ffi.lib().tdg_mg_p1_embedding(dim, kind, degree, out.ctypes.data))
    return out
