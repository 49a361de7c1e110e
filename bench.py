"""Benchmark of the matrix-free DG operator apply (and optionally the block-Jacobi CG solve).

Workload: 3D isotropic elasticity, degree 4, unit cube 32^3 cells x 6 tetrahedra (196,608 tets,
20,643,840 DOF), boundary curved by a P2 geometry map, lambda/mu log-normal random fields,
tandem's volume/facet quadrature rules (57 / 19 points).  All inputs are synthetic and seeded.

A step is one FP64 operator apply y = A x over the whole mesh.  `value` is DOF/s over all ranks
(each rank runs an independent replica: the apply has no data-path collective), timed with CUDA
events between barriers on the launching stream, max over ranks.  `e2e` is the same metric
through the C ABI with host buffers: pinned host x -> device, apply, device -> pinned host y,
every step.  `cpu_baseline` times the CPU restatement of tandem's element-centric apply (the
oracle, OpenMP over all host cores) on a bounded sample of the same elements.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 32] [--solve]

Further workloads (one JSON line each): `--workload poisson` (2D Poisson p4, 64x64x2 GenMesh),
`--workload batch` (uneven batch of independent 2D elasticity solves, FP64 vs mixed),
`--workload gf` (discrete Green's function columns, FP64 vs mixed, RHS/s) and
`--workload adjoint` (Lame gradient time and its check against finite differences).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DOF/s of matrix-free DG apply; solve time to 1e-10 rel. residual, mixed vs FP64"
FP64_PROBES = ("dfma", "dmma_m8n8k4", "dmma_m16n8k4", "dmma_m16n8k8", "dmma_m16n8k16", "dfma_and_dmma")
# solve arms: (name, solve precision, preconditioner precision, preconditioner).  Block Jacobi:
# FP64 CG; mixed = FP64 recurrence around the FP32 tensor-core operator with FP32 (or FP64) block
# inverses; fp32_recurrence = FP32 vectors and recurrence with FP64 reliable updates.  Multigrid:
# p-multigrid (tandem's mg_cheby configuration, continuous P1 coarse space) under flexible CG,
# all FP64, or mixed = FP32 arithmetic in the finest level's smoother and the outer operator.
# The fifth entry is the Krylov method: CG, or flexible GMRES(30) as tandem's multigrid
# configuration runs it (examples/options/mg_cheby.cfg: -ksp_type fgmres).
BJ_ARMS = (("fp64", 0, 0, "bjacobi", "cg"), ("mixed", 2, 1, "bjacobi", "cg"), ("mixed_fp64_pc", 2, 0, "bjacobi", "cg"),
           ("fp32_recurrence", 1, 1, "bjacobi", "cg"))
# mg_tf32: the mixed solve (3xTF32 operator in the FP64 refinement) whose smoother runs the
# finest level's applies in one TF32 pass (precision 3, TDG_TF32)
MG_ARMS = (("mg_fp64", 0, 0, "mg", "cg"), ("mg_mixed", 2, 2, "mg", "cg"), ("mg_tf32", 2, 3, "mg", "cg"))
GMRES_ARMS = (("mg_fgmres_fp64", 0, 0, "mg", "fgmres"), ("mg_fgmres_mixed", 2, 2, "mg", "fgmres"),
              ("mg_fgmres_tf32", 2, 3, "mg", "fgmres"))
SOLVE_ARMS = BJ_ARMS + MG_ARMS + GMRES_ARMS
# the default cube leg: tandem's FP64 configuration (block-Jacobi CG), the two multigrid CG arms
# and multigrid FGMRES in FP64 (tandem's multigrid configuration)
DEFAULT_CUBE_ARMS = BJ_ARMS[:1] + MG_ARMS + GMRES_ARMS[:1]


def select_arms(args, default=SOLVE_ARMS):
    """The solve arms a leg runs: --arms (comma-separated names) or the leg's default set."""
    if not args.arms:
        return default
    want = args.arms.split(",")
    unknown = set(want) - {a[0] for a in SOLVE_ARMS}
    if unknown:
        raise SystemExit(f"unknown solve arms {sorted(unknown)}")
    return tuple(a for a in SOLVE_ARMS if a[0] in want)


# Chebyshev steps per smoothing of the multigrid arms (tandem's mg_cheby.cfg uses 10, the library's
# default; 6 measured faster on the C2 solve in both precisions: 7.48 / 6.19 s against 8.63 / 6.90 s)
MG_SMOOTH_ITS = 6


def prepare_arm(op, pcp: int, pc: str) -> float:
    """Sets up the arm's preconditioner and selects it; returns the set-up wall seconds."""
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    if pc == "mg":
        op.mg_setup(smooth_precision=pcp, smooth_its=MG_SMOOTH_ITS)
        op.set_preconditioner("mg")
    else:
        op.set_preconditioner("bjacobi")
        op.bjacobi_setup(pcp)
    torch.cuda.synchronize()
    return time.perf_counter() - t0


def add_speedups(res: dict, key: str = "seconds") -> None:
    """speedup_vs_fp64 (block-Jacobi FP64 CG, tandem's default solver configuration) for every other
    arm, and speedup_vs_mg_fp64 for the mixed multigrid arms."""
    for name, r in res.items():
        if name != "fp64" and "fp64" in res:
            r["speedup_vs_fp64"] = res["fp64"][key] / r[key]
    for name in ("mg_mixed", "mg_tf32"):
        if "mg_fp64" in res and name in res:
            res[name]["speedup_vs_mg_fp64"] = res["mg_fp64"][key] / res[name][key]
KERNEL_NAMES = {"tensor": "apply_mma_kernel<Shape<3,4,Elasticity>> (FP64 mma.sync m8n8k4, element-centric)",
                "face": "vol_mma_kernel + face_mma_kernel<Shape<3,4,Elasticity>> (FP64 mma.sync m8n8k4, "
                        "face-centric; roofline over both launches of one apply)",
                "face2": "vol2_kernel + face2_kernel<Shape<3,4,Elasticity>> (FP64 mma.sync m8n8k4, face-centric, "
                         "cp.async double-buffered coefficient blocks, tile-ordered geometry; roofline over both "
                         "launches of one apply)",
                "simt": "apply_kernel<Shape<3,4,Elasticity>, double> (SIMT)"}


def launches_per_apply(tune):
    """Kernel launches of one apply in the fastest configuration of an autotune list: the
    face-centric families launch a volume and a facet kernel, the others one kernel."""
    best = min(tune, key=lambda e: e["ms"] if e.get("ms") is not None else 0.0)
    return 2 if best["family"] in ("face", "face2", "tc05") else 1


def fp64_peaks(stream) -> dict:
    """Measured FP64 throughput of this GPU (tdg_probe_fp64_peak): every FP64 path (CUDA-core FMA
    and the tensor pipe's f64 mma.sync shapes) at 2 and 4 CTAs of 256 threads per SM, best of three
    20 ms launches each.  The roofline denominator of the FP64 apply is the largest of them."""
    import ctypes as C
    from tandem_b200 import _ffi
    out = {}
    for kind, name in enumerate(FP64_PROBES):
        best = 0.0
        for ctas in (2, 4):
            v = C.c_double(0.0)
            _ffi.check(_ffi.lib().tdg_probe_fp64_peak(kind, ctas, C.c_void_p(stream.cuda_stream), C.byref(v)))
            best = max(best, v.value)
        out[name] = best
    return out


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def tandem_quadrature(dim: int, degree: int):
    """tandem's volRule / fctRule (simplexQuadratureRule of order 2N+1), from the golden fixture
    generated by tandem's own quadrature sources."""
    from tandem_b200.operator import Quadrature
    rules = json.loads((ROOT / "tests" / "golden" / "quadrature.json").read_text())["auto"]
    order = 2 * degree + 1
    v, f = rules[f"{dim}:{order}"], rules[f"{dim - 1}:{order}"]
    return Quadrature(np.array(v["points"]).reshape(-1, dim), np.array(v["weights"]),
                      np.array(f["points"]).reshape(-1, dim - 1), np.array(f["weights"]))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 15.0 and self.proc.poll() is None:
                time.sleep(0.05)  # start sampling before the timed region, never inside it
            self.mark = len(self.lines)
        except (OSError, ValueError):
            self.proc = None
        return self

    def start_timed(self):
        self.mark = len(self.lines)

    def stop_timed(self):
        self.end = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        lines = self.lines[getattr(self, "mark", 0):getattr(self, "end", len(self.lines))] or self.lines[-3:]
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) != 7:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), float(parts[2]), parts[3:]))
            except ValueError:
                continue
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[3]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": max(r[1] for r in rows),
                "power_w_max": max(r[2] for r in rows), "samples": len(rows), "reasons": reasons}


def cpu_apply_sample(wl, target_s: float, threads: int, max_elements: int | None = None, full_max_s: float = 0.0):
    """Times the oracle's element-centric apply on a contiguous slice of elements: the whole mesh
    when one apply is estimated to take at most full_max_s seconds, else about target_s seconds of
    elements from the middle third on."""
    from oracle import Oracle
    orc = getattr(wl, "orc", None) or Oracle(wl.mesh, wl.degree, wl.kind, wl.quad)
    orc.set_material(wl.c0, wl.c1)
    x = np.random.default_rng(1).standard_normal(orc.ndof)
    y = np.zeros_like(x)
    E = orc.E
    e0 = E // 3
    n = min(512, E - e0)
    orc.apply_range(e0, e0 + n, x, y)  # first touch
    t = time.perf_counter()
    orc.apply_range(e0, e0 + n, x, y)
    dt = time.perf_counter() - t
    per_el = max(dt / n, 1e-7)
    if per_el * E <= full_max_s:
        return orc, x, y, 0, E
    n = int(min(E - e0, max(n, target_s / per_el)))
    if max_elements:
        n = min(n, max_elements)
    return orc, x, y, e0, n


def cube_config(name: str, elements: int, dofs: int, nq_vol: int, nq_fct: int, world: int) -> dict:
    """The `config` of the default (C2 cube) leg; both arms print the same one."""
    return {"workload": name, "elements": int(elements), "dofs": int(dofs), "degree": 4,
            "quadrature": f"tandem volRule {nq_vol} / fctRule {nq_fct} points",
            "l2": "inputs larger than L2 (x, y 165 MB each, geometry 2.8 GB per apply)",
            "parallelism": f"replicas x{world}",
            "solve": "to 1e-10 rel. FP64 residual; fp64 = block-Jacobi CG (tandem's default solver); "
                     "multigrid arms: logarithmic p1-p2-p4, continuous P1 coarse space, "
                     f"{MG_SMOOTH_ITS} Chebyshev steps per smoothing, flexible CG or FGMRES(30)"}


def cpu_solve_sample(wl, iterations: int = 20) -> dict:
    """tandem's algorithm on the host (the oracle's element-centric apply and block-Jacobi CG,
    OpenMP on every core) for `iterations` CG iterations of the workload's system: seconds per
    iteration, after one call that builds the block inverses (timed apart)."""
    from oracle import Oracle
    orc = Oracle(wl.mesh, wl.degree, wl.kind, wl.quad)
    orc.set_material(wl.c0, wl.c1)
    b = orc.rhs(wl.force, wl.bc)
    t0 = time.perf_counter()
    orc.cg(b, rtol=1e-10, maxit=1)  # assembles and inverts the diagonal blocks
    t1 = time.perf_counter()
    _, st = orc.cg(b, rtol=1e-10, maxit=iterations)
    t2 = time.perf_counter()
    return {"seconds_per_iteration": (t2 - t1) / max(st["iterations"], 1), "iterations_sampled": st["iterations"],
            "pc_setup_seconds": t1 - t0, "cores": os.cpu_count(), "kind": "port"}


def oracle_elasticity_cube(n: int, degree: int):
    """The cube workload of elasticity_cube (same mesh, curved boundary, material fields and seeds)
    built with the oracle alone: geometry nodes from the oracle's reference tables, quadrature-point
    coordinates from the oracle, so the CPU arm neither loads the product library nor touches a GPU."""
    from types import SimpleNamespace
    from oracle import Oracle, Tables
    from tandem_b200 import mesh as M
    from tandem_b200.scenarios import RandomField
    quad = tandem_quadrature(3, degree)
    m = M.build(M.cube_mesh(n), degree, curve=M.box_boundary_surface(0.02), tables=Tables)
    orc = Oracle(m, degree, 1, quad)
    X = orc.volume_coords()
    c0, c1 = RandomField(3, 2024, ell=0.2)(X), RandomField(3, 2025, ell=0.2)(X)
    name = (f"3D isotropic elasticity p{degree}, unit cube {n}^3 x 6 tets ({m.num_elements:,}), curved P2 boundary, "
            "log-normal lambda/mu")
    return SimpleNamespace(name=name, mesh=m, quad=quad, kind=1, degree=degree, c0=c0, c1=c1, orc=orc)


def run_reference(args):
    """CPU reference arm: tandem's element-centric apply restated (the oracle), all host cores,
    each step the whole mesh (a slice of its elements where one apply would take over 6 s)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = oracle_elasticity_cube(args.n, 4)
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    orc, x, y, e0, n = cpu_apply_sample(wl, target_s=3.0, threads=threads, full_max_s=6.0)
    for _ in range(args.warmup):
        orc.apply_range(e0, e0 + n, x, y)
    t = time.perf_counter()
    for _ in range(args.steps):
        orc.apply_range(e0, e0 + n, x, y)
    dt = time.perf_counter() - t
    dofs = n * orc.bs * args.steps
    val = dofs / dt
    sample = (f"all {orc.E:,} elements per step" if n == orc.E else f"{n:,} of {orc.E:,} elements per step") + \
        f" (element-centric FP64 apply, OpenMP on {threads} host threads)"
    out = {"metric": METRIC, "value": val, "unit": "DOF/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded mesh, random-field material)",
           "impl": "reference",
           "config": cube_config(wl.name, orc.E, orc.ndof, orc.Nq, orc.nq, args.gpus),
           "cpu_baseline": {"value": val, "unit": "DOF/s", "cores": threads, "kind": "port", "sample": sample},
           "e2e": {"value": val, "unit": "DOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def host_link_bandwidth(hx, hy, stream, reps=3):
    """Host link bandwidth with pinned buffers: one direction alone and both directions at once
    (the copy-in and copy-out streams of the host-buffer apply run together).  Best of `reps`."""
    import torch
    dx = torch.empty_like(hx, device="cuda")
    dy = torch.zeros_like(hy, device="cuda")
    other = torch.cuda.Stream()
    nbytes = hx.numel() * hx.element_size()

    def timed(fn):
        best = float("inf")
        for _ in range(reps + 1):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b))
        return best

    def h2d():
        with torch.cuda.stream(stream):
            dx.copy_(hx, non_blocking=True)

    def both():
        other.wait_stream(stream)
        with torch.cuda.stream(stream):
            dx.copy_(hx, non_blocking=True)
        with torch.cuda.stream(other):
            hy.copy_(dy, non_blocking=True)
        stream.wait_stream(other)

    ms1, ms2 = timed(h2d), timed(both)
    return {"h2d_gbs": nbytes / (ms1 * 1e6), "both_gbs": 2 * nbytes / (ms2 * 1e6)}


def run_ours(args):
    import torch
    import torch.distributed as dist
    from tandem_b200.operator import FP32, FP64, MIXED, TF32
    from tandem_b200.workloads import elasticity_cube

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    wl = elasticity_cube(args.n, 4, tandem_quadrature(3, 4))
    op = wl.op
    n = op.ndof
    stream = torch.cuda.current_stream()
    g = torch.Generator(device="cuda").manual_seed(1234 + rank)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    y = torch.empty_like(x)

    # ---- measured FP64 peaks (roofline denominator), the fastest FP64 launch configuration for
    # this mesh, then the device-resident apply ----
    probes = fp64_peaks(stream)
    if args.family:
        # a fixed launch configuration (profiling runs): no autotuner candidates before the apply
        op.set_apply_config(FP64, args.family, args.ctas, args.tile)
        tune64 = [{"family": args.family, "ctas_per_sm": args.ctas, "tile": args.tile, "ms": None}]
    else:
        tune64 = op.autotune(FP64, stream=stream)
    best64 = min(tune64, key=lambda e: e["ms"] or 0.0)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        for _ in range(args.warmup):
            op.apply(x, y, FP64, stream=stream)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        clk.start_timed()
        ev0.record(stream)
        for _ in range(args.steps):
            op.apply(x, y, FP64, stream=stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        clk.stop_timed()
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1)) / args.steps
    value = world * n / (ms * 1e-3)

    # ---- end to end through the C ABI with pinned host buffers (tdg_apply_host): every step copies
    # x in from pinned host memory, applies and copies y back to host memory; the copies of
    # neighbouring steps overlap the apply (two device buffer pairs, three streams) ----
    hx = torch.randn(n, dtype=torch.float64, generator=torch.Generator().manual_seed(99)).pin_memory()
    hy = torch.empty(n, dtype=torch.float64).pin_memory()
    op.apply_host(hx, hy, FP64, count=max(2, args.warmup), stride=0, stream=stream)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    op.apply_host(hx, hy, FP64, count=args.steps, stride=0, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1)) / args.steps
    link = host_link_bandwidth(hx, hy, stream)
    e2e = {"value": world * n / (ms_e2e * 1e-3), "unit": "DOF/s", "h2d_bytes_per_step": n * 8,
           "d2h_bytes_per_step": n * 8, "ms_per_step": ms_e2e,
           "api": "tdg_apply_host: per step H2D of x from pinned host memory, apply, D2H of y; the copies "
                  "of neighbouring steps overlap the apply (two device buffer pairs, three streams)",
           "link": link, "link_bound_ms": 2 * n * 8 / (link["both_gbs"] * 1e6)}

    # ---- FP32 apply (inner operator of the mixed-precision solve), fastest configuration ----
    if args.family32:
        op.set_apply_config(FP32, args.family32, args.ctas)
        tune32 = [{"family": args.family32, "ctas_per_sm": args.ctas, "ms": 0.0}]
    else:
        tune32 = op.autotune(FP32, stream=stream)
    best32 = min(tune32, key=lambda e: e["ms"])
    x32, y32 = x.float(), torch.empty(n, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        op.apply(x32, y32, FP32, stream=stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        op.apply(x32, y32, FP32, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms32 = max_over_ranks(e0.elapsed_time(e1)) / args.steps
    # the same operator on FP64 vectors: 3xTF32 (TDG_MIXED, the mixed solve's operator) and one TF32
    # pass (TDG_TF32, the mixed multigrid smoother's), with their deviation from the FP64 apply
    y64 = torch.empty_like(x)
    op.apply(x, y64, FP64, stream=stream)
    tf = {}
    for name, prec in (("mixed", MIXED), ("tf32", TF32)):
        yt = torch.empty_like(x)
        for _ in range(args.warmup):
            op.apply(x, yt, prec, stream=stream)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            op.apply(x, yt, prec, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        mst = max_over_ranks(e0.elapsed_time(e1)) / args.steps
        tf[name] = {"ms_per_step": mst, "value": world * n / (mst * 1e-3), "unit": "DOF/s",
                    "rel_diff_vs_fp64": float(torch.norm(yt - y64) / torch.norm(y64))}
        del yt
    del y64

    solve = None
    arms = select_arms(args) if args.solve or args.arms else (() if args.no_solve else DEFAULT_CUBE_ARMS)
    if arms:
        b = torch.as_tensor(op.rhs(wl.force, wl.bc), device="cuda")
        solve = {}
        x_first = None
        for name, prec, pcp, pc, method in arms:
            setup_s = max_over_ranks(prepare_arm(op, pcp, pc))
            xs = torch.zeros_like(b)
            st = op.solve(b, xs, precision=prec, rtol=1e-10, max_iterations=args.max_iterations, check=False,
                          method=method)
            solve[name] = {"seconds": max_over_ranks(st["seconds"]), "iterations": st["iterations"],
                           "reliable_updates": st["outer"], "fp64_continuation_iterations": st["fp64_iterations"],
                           "rel_residual": st["rel_residual"], "pc_setup_seconds": setup_s}
            if x_first is None:
                x_first, first = xs.clone(), name
            else:
                solve[name][f"rel_diff_vs_{first}"] = float(torch.norm(xs - x_first) / torch.norm(x_first))
        op.set_preconditioner("bjacobi")
        add_speedups(solve)
        if args.solve and not args.no_cpu and args.n <= 16 and rank == 0:
            # host baseline: a bounded sample of block-Jacobi CG iterations, extrapolated to the
            # device's FP64 block-Jacobi iteration count (the full host solve takes tens of minutes)
            cs = cpu_solve_sample(wl)
            if "fp64" in solve:
                cs["extrapolated_seconds"] = cs["seconds_per_iteration"] * solve["fp64"]["iterations"]
                cs["extrapolated_to_iterations"] = solve["fp64"]["iterations"]
            solve["cpu_block_jacobi_sample"] = cs

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    hbm, peak_kind = peaks()
    bytes_apply = op.bytes_apply(FP64)
    flops_apply = op.flops_apply()
    achieved = bytes_apply / (ms * 1e-3) / 1e9
    tflops = flops_apply / (ms * 1e-3) / 1e12
    # the denominator: the best single FP64 path (the concurrent probe is reported beside it)
    fp64_peak = max(v for k, v in probes.items() if k != "dfma_and_dmma")
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get(f"apply_fp64_{best64['family']}_cube{args.n}")
    # 3D p4 elasticity runs at ~15 FLOP/B, right of the FP64 ridge (~40 TF/s over ~6.5 TB/s):
    # the FP64 pipe binds, HBM is reported beside it
    roofline = {"bound": "fp64", "achieved": tflops, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": tflops / fp64_peak, "traffic": traffic,
                "peak_source": "measured in this run (tdg_probe_fp64_peak, best FP64 path: "
                               + max((k for k in probes if k != "dfma_and_dmma"), key=probes.get) + ")",
                "fp64_probes_tflops": probes,
                "kernel": KERNEL_NAMES[best64["family"]],
                "algorithmic_flops_per_launch": flops_apply, "algorithmic_bytes_per_launch": bytes_apply,
                "hbm": {"achieved_gbs": achieved, "peak_gbs": hbm, "frac": achieved / hbm,
                        "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"}}
    cpu = None
    if world == 1 and not args.no_cpu:
        threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        orc, xc, yc, ce0, cn = cpu_apply_sample(wl, target_s=2.0, threads=threads)
        reps, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < args.cpu_seconds:
            orc.apply_range(ce0, ce0 + cn, xc, yc)
            reps += 1
        dt = time.perf_counter() - t0
        cpu = {"value": reps * cn * orc.bs / dt, "unit": "DOF/s", "cores": threads, "kind": "port",
               "sample": f"{reps} x {cn:,} of {orc.E:,} elements (element-centric FP64 apply, OpenMP, {dt:.1f} s)"}
    out = {"metric": METRIC, "value": value, "unit": "DOF/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded mesh, random-field material)",
           "config": cube_config(wl.name, op.E, n, op.Nq, op.nq, world),
           "clocks": clk.summary(), "e2e": e2e,
           "gpu_launches": args.steps * launches_per_apply([best64]),
           "apply_config": best64, "autotune": tune64,
           "roofline": roofline, "cpu_baseline": cpu,
           "fp32_apply": {"value": world * n / (ms32 * 1e-3), "unit": "DOF/s", "ms_per_step": ms32,
                          "config": best32},
           "fp64_vector_applies": tf,
           "solve": solve}
    print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


def _event_time(fn, steps: int, warmup: int, stream) -> float:
    """ms per call of fn() on `stream`, CUDA events, after warm-up."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _init_ranks():
    """(world, rank) of a torchrun launch, with an nccl process group on this rank's GPU (world > 1)."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    return world, rank


def _timed_max(fn, world):
    """Seconds of fn() on this rank (CUDA events on the current stream, barriers around), max over ranks."""
    import torch
    import torch.distributed as dist
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1) / 1e3], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item()), out


def run_batch_sharded(args, world, rank):
    """The uneven batch over the ranks: problems assigned longest-processing-time first by element
    count (sharding.lpt_assign), each rank solving its share as one segmented solve; no data-path
    collective.  value = DOF of the whole batch / the slowest rank's solve time."""
    import torch
    import torch.distributed as dist
    from tandem_b200.operator import solve_segmented
    from tandem_b200.sharding import lpt_assign
    from tandem_b200.workloads import uneven_batch, uneven_batch_cells
    cells = uneven_batch_cells(args.count)
    sizes = 2 * cells.astype(np.int64) ** 2
    mine = lpt_assign(sizes, world)[rank]
    b = uneven_batch(args.count, 4, tandem_quadrature(2, 4), problems=mine)
    op = b.op
    rhs = torch.as_tensor(op.rhs(b.force, b.bc), device="cuda")
    arms = select_arms(args, default=MG_ARMS)
    res = {}
    for name, prec, pcp, pc, method in arms:
        setup_s = prepare_arm(op, pcp, pc)
        xs = torch.zeros(op.ndof, dtype=torch.float64, device="cuda")
        secs, (st, rel) = _timed_max(lambda: solve_segmented(op, rhs, xs, b.elem_offsets, precision=prec, rtol=1e-10,
                                                             max_iterations=args.max_iterations, check=False,
                                                             method=method), world)
        worst = torch.tensor([float(np.max(rel))], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(worst, op=dist.ReduceOp.MAX)
        res[name] = {"seconds": secs, "max_rel_residual": float(worst.item()), "pc_setup_seconds": setup_s}
    total_dof = int(sizes.sum()) * 30
    if rank == 0:
        best = min(res, key=lambda k: res[k]["seconds"])
        out = {"metric": "uneven batch solve DOF/s (every problem to 1e-10 rel. residual)",
               "value": total_dof / res[best]["seconds"], "value_arm": best, "unit": "DOF/s", "n_gpus": world,
               "higher_is_better": True, "scaling": "strong", "dtype": "f64", "data": "synthetic (seeded meshes)",
               "config": {"workload": f"{args.count} uneven 2D elasticity problems p4", "dofs": total_dof,
                          "parallelism": f"LPT problem assignment over {world} ranks"},
               "solve": res}
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_gf_sharded(args, world, rank):
    """Green's-function columns over the ranks: contiguous column blocks per rank
    (sharding.column_block), one gather of the column blocks to rank 0 at the end.  value = columns
    / the slowest rank's time (solves and traction of its block)."""
    import torch
    import torch.distributed as dist
    from tandem_b200 import mesh as M
    from tandem_b200.operator import DGOperator, POISSON, Fault, greens_function
    from tandem_b200.sharding import column_block, gather_columns
    m = M.graded_fault_mesh()
    M.topology(m, m.info["boundary_bc"], m.info["interior_bc"])
    M.geometry_nodes(m, 4)
    op = DGOperator(m, 4, POISSON, tandem_quadrature(2, 4))
    op.set_material(np.ones((op.E, op.Nq)))
    fl = Fault(op, M.fault_facets(m), np.array([1.0, 0.0]))
    ncols = fl.ncoef if args.columns <= 0 else min(args.columns, fl.ncoef)
    c0, c1 = column_block(ncols, world, rank)
    res = {}
    for name, prec, pcp, pc, method in select_arms(args, default=MG_ARMS):
        prepare_arm(op, pcp, pc)
        secs, (G, _) = _timed_max(lambda: greens_function(op, fl, precision=prec, rtol=1e-10,
                                                          columns=np.arange(c0, c1), batch=args.batch,
                                                          max_iterations=args.max_iterations, method=method), world)
        full = gather_columns(G, ncols) if world > 1 else G
        res[name] = {"seconds": secs, "rhs_per_s": ncols / secs}
        if rank == 0:
            res[name]["columns_gathered"] = int(full.shape[1])
    if rank == 0:
        best = max(res, key=lambda k: res[k]["rhs_per_s"])
        print(json.dumps({"metric": "Green's function RHS/s (unit-slip columns solved to 1e-10 rel. residual)",
                          "value": res[best]["rhs_per_s"], "value_arm": best, "unit": "RHS/s", "n_gpus": world,
                          "higher_is_better": True, "scaling": "strong", "dtype": "f64",
                          "data": "synthetic graded fault mesh",
                          "config": {"workload": f"2D antiplane Poisson p4, {op.E:,} triangles", "columns": ncols,
                                     "batch": args.batch, "parallelism": f"column blocks over {world} ranks"},
                          "greens_function": res}), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_batch(args):
    """Uneven batch: independent 2D elasticity problems in one block-diagonal operator; apply
    throughput after autotuning, then FP64 and mixed segmented solves to 1e-10 per problem."""
    import torch
    from tandem_b200.operator import FP32, FP64, solve_segmented
    from tandem_b200.workloads import uneven_batch

    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    b = uneven_batch(args.count, 4, tandem_quadrature(2, 4))
    setup_s = time.perf_counter() - t0
    op, n = b.op, b.op.ndof
    stream = torch.cuda.current_stream()
    tune = {"fp64": op.autotune(FP64), "fp32": op.autotune(FP32)}
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=torch.Generator(device="cuda").manual_seed(3))
    y = torch.empty_like(x)
    with ClockSampler(0) as clk:
        clk.start_timed()
        ms64 = _event_time(lambda: op.apply(x, y, FP64, stream=stream), args.steps, args.warmup, stream)
        clk.stop_timed()
    x32, y32 = x.float(), torch.empty(n, dtype=torch.float32, device="cuda")
    ms32 = _event_time(lambda: op.apply(x32, y32, FP32, stream=stream), args.steps, args.warmup, stream)
    rhs_h = torch.as_tensor(op.rhs(b.force, b.bc)).pin_memory()
    solve = {}
    sol = {}
    arms = select_arms(args)
    for name, prec, pcp, pc, method in arms:
        setup_s = prepare_arm(op, pcp, pc)
        rhs = rhs_h.to("cuda", non_blocking=True)
        xs = torch.zeros(n, dtype=torch.float64, device="cuda")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        rhs = rhs_h.to("cuda", non_blocking=True)
        st, rel = solve_segmented(op, rhs, xs, b.elem_offsets, precision=prec, rtol=1e-10,
                                  max_iterations=args.max_iterations, check=False, method=method)
        xh = xs.to("cpu")
        e1.record(stream)
        torch.cuda.synchronize()
        sol[name] = xs
        solve[name] = {"seconds": st["seconds"], "e2e_seconds": e0.elapsed_time(e1) / 1e3,
                       "iterations": st["iterations"], "reliable_updates": st["outer"],
                       "fp64_continuation_iterations": st["fp64_iterations"],
                       "max_rel_residual": float(np.max(rel)), "problems_converged": int(np.sum(rel <= 1e-10)),
                       "rel_residual_per_problem": [float(v) for v in rel], "pc_setup_seconds": setup_s}
        del xh
    op.set_preconditioner("bjacobi")
    for name, _, _, _, _ in arms[1:]:
        d = []
        for i in range(args.count):
            sl = slice(int(b.elem_offsets[i]) * op.bs, int(b.elem_offsets[i + 1]) * op.bs)
            ref = sol[arms[0][0]][sl]
            d.append(float(torch.norm(sol[name][sl] - ref) / torch.norm(ref)))
        solve[name][f"max_rel_diff_vs_{arms[0][0]}_per_problem"] = max(d)
    add_speedups(solve)
    out = {"metric": METRIC, "value": n / (ms64 * 1e-3), "unit": "DOF/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms64, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded meshes, random-field material and force)",
           "config": {"workload": b.name, "problems": args.count, "elements": int(op.E), "dofs": int(n),
                      "sizes": [int(v) for v in b.sizes], "setup_seconds": setup_s},
           "clocks": clk.summary(), "gpu_launches": args.steps * launches_per_apply(tune["fp64"]), "autotune": tune,
           "fp32_apply": {"value": n / (ms32 * 1e-3), "unit": "DOF/s", "ms_per_step": ms32},
           "solve": solve,
           "solve_dof_per_s": {k: n / v["seconds"] for k, v in solve.items() if isinstance(v, dict)}}
    print(json.dumps(out), flush=True)


def run_gf(args):
    """Discrete Green's function of a 2D antiplane (Poisson) fault problem: `columns` unit-slip
    right-hand sides solved as batched multi-RHS CG launches of `batch` columns, FP64 and mixed;
    RHS/s and the difference of the mixed columns from the FP64 ones."""
    import torch
    from tandem_b200 import mesh as M
    from tandem_b200.operator import DGOperator, FP32, FP64, POISSON, Fault, greens_function

    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    m = M.graded_fault_mesh()
    M.topology(m, m.info["boundary_bc"], m.info["interior_bc"])
    M.geometry_nodes(m, 4)
    op = DGOperator(m, 4, POISSON, tandem_quadrature(2, 4))
    op.set_material(np.ones((op.E, op.Nq)))
    fl = Fault(op, M.fault_facets(m), np.array([1.0, 0.0]))
    setup_s = time.perf_counter() - t0
    ncols = fl.ncoef if args.columns <= 0 else min(args.columns, fl.ncoef)
    cols = np.arange(ncols)
    tune = {"fp64": op.autotune(FP64, nrhs=min(args.batch, ncols)),
            "fp32": op.autotune(FP32, nrhs=min(args.batch, ncols))}
    res, Gs = {}, {}
    arms = select_arms(args)
    for name, prec, pcp, pc, method in arms:
        setup_s = prepare_arm(op, pcp, pc)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        G, stats = greens_function(op, fl, precision=prec, rtol=1e-10, columns=cols, batch=args.batch,
                                   max_iterations=args.max_iterations, method=method)
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
        Gs[name] = G
        res[name] = {"seconds": wall, "rhs_per_s": ncols / wall, "batches": len(stats),
                     "iterations": [s["iterations"] for s in stats],
                     "reliable_updates": [s["outer"] for s in stats],
                     "fp64_continuation_iterations": [s["fp64_iterations"] for s in stats],
                     "max_rel_residual": max(s["rel_residual"] for s in stats), "pc_setup_seconds": setup_s}
    op.set_preconditioner("bjacobi")
    first = arms[0][0]
    for name, _, _, _, _ in arms[1:]:
        diff = torch.norm(Gs[name] - Gs[first], dim=0) / torch.norm(Gs[first], dim=0)
        res[name][f"max_column_rel_diff_vs_{first}"] = float(diff.max())
    add_speedups(res)
    best = max(res, key=lambda k: res[k]["rhs_per_s"])
    out = {"metric": "Green's function RHS/s (unit-slip columns solved to 1e-10 rel. residual)",
           "value": res[best]["rhs_per_s"], "value_arm": best, "unit": "RHS/s", "n_gpus": 1,
           "higher_is_better": True, "dtype": "f64 (mixed: fp32 inner)", "data": "synthetic graded fault mesh",
           "config": {"workload": f"2D antiplane Poisson p4, {op.E:,} triangles graded toward a 60 deg fault of "
                                  f"{fl.nfault} facets ({fl.ncoef} fault basis functions)",
                      "columns": int(ncols), "batch": args.batch, "dofs_per_rhs": int(op.ndof),
                      "setup_seconds": setup_s},
           "autotune": tune, "greens_function": res}
    print(json.dumps(out), flush=True)


def run_poisson(args):
    """2D Poisson p4 on tandem's GenMesh<2> 64 x 64 x 2 triangles (K = 1, sin sin MMS): apply
    throughput (FP64 / FP32) and the FP64 vs mixed CG solve to 1e-10."""
    import torch
    from tandem_b200.operator import FP32, FP64
    from tandem_b200.workloads import poisson_square

    torch.cuda.set_device(0)
    wl = poisson_square(args.square, 4, tandem_quadrature(2, 4))
    op, n = wl.op, wl.op.ndof
    stream = torch.cuda.current_stream()
    tune = {"fp64": op.autotune(FP64), "fp32": op.autotune(FP32)}
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=torch.Generator(device="cuda").manual_seed(5))
    y = torch.empty_like(x)
    ms64 = _event_time(lambda: op.apply(x, y, FP64, stream=stream), args.steps, args.warmup, stream)
    x32, y32 = x.float(), torch.empty(n, dtype=torch.float32, device="cuda")
    ms32 = _event_time(lambda: op.apply(x32, y32, FP32, stream=stream), args.steps, args.warmup, stream)
    b = torch.as_tensor(op.rhs(wl.force, wl.bc), device="cuda")
    solve, sol = {}, {}
    arms = select_arms(args)
    for name, prec, pcp, pc, method in arms:
        setup_s = prepare_arm(op, pcp, pc)
        xs = torch.zeros_like(b)
        st = op.solve(b, xs, precision=prec, rtol=1e-10, max_iterations=args.max_iterations, check=False,
                      method=method)
        sol[name] = xs
        solve[name] = {"seconds": st["seconds"], "iterations": st["iterations"], "reliable_updates": st["outer"],
                       "fp64_continuation_iterations": st["fp64_iterations"], "rel_residual": st["rel_residual"],
                       "pc_setup_seconds": setup_s}
        if name != arms[0][0]:
            ref = sol[arms[0][0]]
            solve[name][f"rel_diff_vs_{arms[0][0]}"] = float(torch.norm(xs - ref) / torch.norm(ref))
    op.set_preconditioner("bjacobi")
    add_speedups(solve)
    cpu_solve = None
    if not args.no_cpu:
        # tandem's algorithm on the host: the oracle's element-centric apply and block-Jacobi CG
        # (OpenMP on every host core), the same system to the same residual target
        from oracle import Oracle
        orc = Oracle(wl.mesh, wl.degree, wl.kind, wl.quad)
        orc.set_material(wl.c0, wl.c1)
        bh = orc.rhs(wl.force, wl.bc)
        c0 = time.perf_counter()
        _, cst = orc.cg(bh, rtol=1e-10, maxit=args.max_iterations)
        cpu_s = time.perf_counter() - c0
        cpu_solve = {"seconds": cpu_s, "iterations": cst["iterations"], "rel_residual": cst["rel_residual"],
                     "cores": os.cpu_count(), "kind": "port",
                     "gpu_speedup": {k: cpu_s / v["seconds"] for k, v in solve.items()}}
    out = {"metric": METRIC, "value": n / (ms64 * 1e-3), "unit": "DOF/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms64, "higher_is_better": True, "dtype": "f64",
           "cpu_solve": cpu_solve,
           "data": "synthetic (tandem GenMesh<2>, sin sin manufactured solution)",
           "config": {"workload": wl.name, "elements": int(op.E), "dofs": int(n),
                      "l2": "L2-resident (14 MB per apply)"},
           "gpu_launches": args.steps * launches_per_apply(tune["fp64"]), "autotune": tune,
           "fp32_apply": {"value": n / (ms32 * 1e-3), "unit": "DOF/s", "ms_per_step": ms32}, "solve": solve}
    print(json.dumps(out), flush=True)


def run_adjoint(args):
    """Lame gradient of a point misfit on the 16^3 x 6 curved tet mesh (degree 4, per-element
    lambda, mu ~ U[0.5, 2]): time of one gradient (forward solve, adjoint solve, gradient kernel)
    and the check against central finite differences on `fd_elements` random elements (lambda_e
    and mu_e separately, relative step --fd-step).  Each FD side solves for the correction
    A(theta') du = b(theta') - A(theta') u0 from the converged u0 and takes the misfit change
    J(u0 + du) - J(u0) = r0 . P du + |P du|^2 / 2 (r0 = P u0 - d), so neither the solve tolerance
    nor the size of J(u0) cancels in the difference."""
    import torch
    from tandem_b200 import mesh as M
    from tandem_b200.adjoint import LameProblem, PointObservation, lame_solve
    from tandem_b200.operator import DGOperator, ELASTICITY, FP32, FP64
    from tandem_b200.scenarios import ElasticityCosine

    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    m = M.build(M.cube_mesh(args.adj_n), 4, curve=M.box_boundary_surface(0.02))
    op = DGOperator(m, 4, ELASTICITY, tandem_quadrature(3, 4))
    X, Xf = op.volume_coords(), op.facet_coords()
    sc = ElasticityCosine(3)
    f = np.ascontiguousarray(np.moveaxis(sc.force(X), -1, 1))
    g = np.ascontiguousarray(np.moveaxis(sc.solution(Xf), -1, 1))
    rng = np.random.Generator(np.random.PCG64(args.seed))
    lam0, mu0 = rng.uniform(0.5, 2.0, op.E), rng.uniform(0.5, 2.0, op.E)
    rng1 = np.random.Generator(np.random.PCG64(args.seed + 1))
    lam_t = lam0 * (1.0 + 0.1 * rng1.uniform(-1.0, 1.0, op.E))
    mu_t = mu0 * (1.0 + 0.1 * rng1.uniform(-1.0, 1.0, op.E))
    pts = np.random.Generator(np.random.PCG64(args.seed + 2)).uniform(0.1, 0.9, size=(512, 3))
    P = PointObservation(m, 4, pts)
    pb = LameProblem(op, f, g, rtol=args.grad_rtol, precision=FP64, preconditioner=args.adj_pc)
    d = P.apply(pb.forward(lam_t, mu_t)).detach()
    setup_s = time.perf_counter() - t0

    lam = torch.tensor(lam0, dtype=torch.float64, requires_grad=True)
    mu = torch.tensor(mu0, dtype=torch.float64, requires_grad=True)
    pb.set_parameters(lam0, mu0)
    pb.last_stats.clear()
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    u = lame_solve(lam, mu, pb)
    J = 0.5 * torch.sum((P.apply(u) - d) ** 2)
    J.backward()
    torch.cuda.synchronize()
    grad_s = time.perf_counter() - w0
    solves = [dict(iterations=s["iterations"], seconds=s["seconds"], rel_residual=s["rel_residual"])
              for s in pb.last_stats]
    gl, gm = lam.grad.numpy().copy(), mu.grad.numpy().copy()
    u0 = u.detach().clone()

    # central finite differences.  Each side replaces the base material by tdg_update_material,
    # which keeps the base point's preconditioner (the perturbation is one element by a factor
    # 1 +- h), and solves for the correction A(theta') du = b(theta') - A(theta') u0 from the
    # converged u0 to fd_rtol relative to that (O(h)) right-hand side; the minus side starts from
    # -du of the plus side (they agree to O(h^2)).
    from tandem_b200.operator import MIXED
    fd_prec = {"fp64": FP64, "mixed": MIXED}[args.fd_precision]
    sel = np.random.Generator(np.random.PCG64(args.seed + 3)).choice(op.E, size=args.fd_elements, replace=False)
    h = args.fd_step
    r0 = (P.apply(u0) - d).detach()  # misfit residual at the base point
    ones = np.ones((1, op.Nq))
    au = torch.empty_like(u0)
    fd_its = []

    def misfit_pair(e, comp):
        vals, du_prev = [], None
        for sgn in (1.0, -1.0):
            lv, mv = lam0.copy(), mu0.copy()
            (lv if comp == "lambda" else mv)[e] *= 1.0 + sgn * h
            op.update_material(lv[:, None] * ones, mv[:, None] * ones)
            r = torch.as_tensor(op.rhs(f, g), device="cuda")
            op.apply(u0, au)
            r -= au
            du = torch.zeros_like(u0) if du_prev is None else -du_prev
            st = op.solve(r, du, precision=fd_prec, rtol=args.fd_rtol, max_iterations=args.max_iterations,
                          check=False)
            fd_its.append(st["iterations"])
            du_prev = du
            # J(u0 + du) - J(u0) = r0 . P du + |P du|^2 / 2, without the cancellation of J(u0)
            pdu = P.apply(du)  # P is linear
            vals.append(float(torch.sum(r0 * pdu)) + 0.5 * float(torch.sum(pdu * pdu)))
        return vals

    errs = {"lambda": [], "mu": []}
    absd = {"lambda": [], "mu": []}
    scale = {"lambda": 0.0, "mu": 0.0}
    f0 = time.perf_counter()
    for e in sel:
        for comp, grad in (("lambda", gl), ("mu", gm)):
            vals = misfit_pair(e, comp)
            step = h * (lam0[e] if comp == "lambda" else mu0[e])
            fd = (vals[0] - vals[1]) / (2.0 * step)
            errs[comp].append(abs(grad[e] - fd) / abs(fd))
            scale[comp] = max(scale[comp], abs(fd))
            absd[comp].append(abs(grad[e] - fd))
    fd_s = time.perf_counter() - f0
    out = {"metric": "adjoint Lame gradient: seconds per gradient, max relative error vs central FD",
           "value": grad_s, "unit": "s", "higher_is_better": False, "n_gpus": 1, "dtype": "f64",
           "data": "synthetic (per-element U[0.5,2] lambda/mu, 10% perturbed data field, seeded points)",
           "config": {"workload": f"3D elasticity p4, unit cube {args.adj_n}^3 x 6 tets ({op.E:,}), curved P2 boundary, "
                                  f"512 observation points in [0.1,0.9]^3", "dofs": int(op.ndof),
                      "fd_elements": int(args.fd_elements), "fd_step_rel": h, "fd_solve_rtol": args.fd_rtol,
                      "fd_solve_precision": args.fd_precision,
                      "fd_preconditioner": f"{args.adj_pc} of the base point (kept by tdg_update_material)",
                      "gradient_solve_rtol": args.grad_rtol, "gradient_preconditioner": args.adj_pc,
                      "setup_seconds": setup_s},
           "misfit": float(J.detach()), "gradient_solves": solves,
           "fd": {"max_rel_err_lambda": max(errs["lambda"]), "max_rel_err_mu": max(errs["mu"]),
                  "median_rel_err_lambda": float(np.median(errs["lambda"])),
                  "median_rel_err_mu": float(np.median(errs["mu"])),
                  "max_err_rel_to_largest_lambda": max(absd["lambda"]) / scale["lambda"],
                  "max_err_rel_to_largest_mu": max(absd["mu"]) / scale["mu"], "seconds": fd_s,
                  "max_rel_err": max(max(errs["lambda"]), max(errs["mu"])),
                  "solve_iterations_mean": float(np.mean(fd_its))}}
    print(json.dumps(out), flush=True)


def run_vcycle(args):
    """One multigrid V-cycle of the cube workload (logarithmic p1-p2-p4 levels, continuous P1 coarse
    space, --mg-smooth-its Chebyshev steps, FP64) after one warm-up V-cycle, with the CUDA profiler
    range (torch.cuda.profiler start / stop) around the timed one, so that a launch-list capture
    (ncu --profile-from-start off) sees exactly one V-cycle."""
    import torch
    from tandem_b200.operator import FP64
    from tandem_b200.workloads import elasticity_cube

    torch.cuda.set_device(0)
    wl = elasticity_cube(args.n, 4, tandem_quadrature(3, 4))
    op = wl.op
    stream = torch.cuda.current_stream()
    tune = op.autotune(FP64, stream=stream)
    op.mg_setup(smooth_its=MG_SMOOTH_ITS)
    g = torch.Generator(device="cuda").manual_seed(7)
    r = torch.randn(op.ndof, dtype=torch.float64, device="cuda", generator=g)
    z = torch.zeros_like(r)
    op.mg_apply(r, z, stream=stream)
    torch.cuda.synchronize()
    c0 = op.mg_info()["coarse_iterations"]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.profiler.start()
    e0.record(stream)
    op.mg_apply(r, z, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    info = op.mg_info()
    out = {"metric": "multigrid V-cycle time", "value": e0.elapsed_time(e1), "unit": "ms", "higher_is_better": False,
           "n_gpus": 1, "dtype": "f64", "data": "synthetic (seeded mesh, random-field material)",
           "config": {"workload": wl.name, "dofs": int(op.ndof), "levels": info["degrees"],
                      "smooth_its": MG_SMOOTH_ITS, "coarse_space": "continuous P1"},
           "coarse_iterations": info["coarse_iterations"] - c0, "apply_config": min(tune, key=lambda e: e["ms"])}
    print(json.dumps(out), flush=True)


def main():
    global MG_SMOOTH_ITS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=32, help="cube cells per direction")
    ap.add_argument("--solve", action="store_true", help="cube: every solve arm (block Jacobi and multigrid); "
                    "by default only the multigrid arms run")
    ap.add_argument("--no-solve", action="store_true", help="cube: apply only")
    ap.add_argument("--mg-smooth-its", type=int, default=MG_SMOOTH_ITS,
                    help="Chebyshev steps per smoothing in the multigrid solve arms")
    ap.add_argument("--arms", default="", help="comma-separated solve arms to run (default: the leg's set): "
                    + ", ".join(a[0] for a in SOLVE_ARMS))
    ap.add_argument("--max-iterations", type=int, default=30000)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--family", choices=["tensor", "face", "face2", "simt"], default="",
                    help="cube: FP64 apply kernel family to use instead of the autotuner's pick")
    ap.add_argument("--family32", choices=["tensor", "face", "tc05", "simt"], default="",
                    help="cube: FP32 apply kernel family to use instead of the autotuner's pick")
    ap.add_argument("--ctas", type=int, default=2, help="cube: persistent CTAs per SM with --family / --family32")
    ap.add_argument("--tile", type=int, default=0,
                    help="cube: volume points per pass with --family face2 (0 = automatic)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--workload", choices=["cube", "batch", "gf", "poisson", "adjoint", "vcycle"], default="cube",
                    help="cube: the apply benchmark (default); batch: uneven batch of 2D elasticity "
                         "solves; gf: discrete Green's function columns; poisson: 2D Poisson p4 "
                         "64x64x2; adjoint: Lame gradient vs finite differences; vcycle: one multigrid "
                         "V-cycle of the cube inside a profiler range")
    ap.add_argument("--count", type=int, default=48, help="batch: number of problems")
    ap.add_argument("--columns", type=int, default=0, help="gf: columns to solve (0 = all)")
    ap.add_argument("--batch", type=int, default=256, help="gf: right-hand sides per solve")
    ap.add_argument("--square", type=int, default=64, help="poisson: cells per direction")
    ap.add_argument("--adj-n", type=int, default=16, help="adjoint: cube cells per direction")
    ap.add_argument("--fd-elements", type=int, default=64, help="adjoint: elements checked by FD")
    ap.add_argument("--fd-rtol", type=float, default=1e-12, help="adjoint: FD correction solve tolerance")
    ap.add_argument("--fd-step", type=float, default=1e-5, help="adjoint: relative FD step")
    ap.add_argument("--fd-precision", choices=["fp64", "mixed"], default="fp64", help="adjoint: FD solve precision")
    ap.add_argument("--grad-rtol", type=float, default=1e-12, help="adjoint: forward / adjoint solve tolerance")
    ap.add_argument("--adj-pc", choices=["bjacobi", "mg"], default="mg", help="adjoint: gradient solves' preconditioner")
    ap.add_argument("--seed", type=int, default=11)
    args = ap.parse_args()
    MG_SMOOTH_ITS = args.mg_smooth_its
    if args.impl == "reference":
        run_reference(args)
    elif args.workload in ("batch", "gf") and int(os.environ.get("WORLD_SIZE", "1")) > 1:
        world, rank = _init_ranks()
        (run_batch_sharded if args.workload == "batch" else run_gf_sharded)(args, world, rank)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "gf":
        run_gf(args)
    elif args.workload == "poisson":
        run_poisson(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    elif args.workload == "vcycle":
        run_vcycle(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
