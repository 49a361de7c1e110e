"""The C++ binding a tandem maintainer adds (tests/cxx/cuda_dg_operator.h: CudaDGOperator over
AbstractDGOperator, the MatShell apply on VECCUDA arrays, block-Jacobi and multigrid PCSHELL
applies) compiled with g++ against minimal stand-ins for tandem's operator interface and PETSc
(tests/cxx/stub), linked to libtandem_b200.so, and run: on the CPU the construction, sizes and
error paths (exceptions from the library's return codes, PETSC_ERR_LIB from the shell, the
tdg_last_error message); on a GPU MatMult and both PC applies on device arrays against the
oracle (1e-12 for the apply, 1e-10 for the block-Jacobi solve)."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cases import make_mesh, material, mixed_bc_mesh, tandem_quadrature
from tandem_b200 import build as tbuild

HERE = Path(__file__).resolve().parent / "cxx"
ROOT = HERE.parents[1]
BUILD = HERE / "_build"
EXE = BUILD / "glue_driver"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))


def _driver() -> Path:
    lib = tbuild.build()
    srcs = [HERE / "glue_driver.cpp", HERE / "cuda_dg_operator.h", HERE / "stub/petsc/petsc_stub.h",
            HERE / "stub/form/AbstractDGOperator.h", ROOT / "include/tandem_b200.h"]
    if EXE.exists() and all(EXE.stat().st_mtime >= p.stat().st_mtime for p in srcs + [lib]):
        return EXE
    BUILD.mkdir(exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", str(HERE / "stub"), "-I", str(HERE),
           "-I", str(ROOT / "include"), "-I", str(CUDA / "include"), str(HERE / "glue_driver.cpp"), "-o", str(EXE),
           "-L", str(lib.parent), "-ltandem_b200", "-Wl,-rpath,$ORIGIN/../../../tandem_b200/_lib",
           "-L", str(CUDA / "lib64"), "-lcudart", "-Wl,-rpath," + str(CUDA / "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return EXE


def _write_inputs(tmp: Path, mesh, degree: int, kind: int, seed: int = 3):
    from tandem_b200.operator import DGOperator
    q = tandem_quadrature(mesh.dim, degree)
    op = DGOperator(mesh, degree, kind, q)  # for the quadrature-point coordinates of the material
    c0, c1 = material(kind, mesh.dim, op.volume_coords(), True)
    meta = np.array([mesh.dim, degree, mesh.geo_degree, mesh.num_elements, mesh.num_facets, kind], dtype=np.int64)
    arrays = dict(meta=meta, up=mesh.facet_up.astype(np.int64), loc=mesh.facet_local.astype(np.int32),
                  bc=mesh.facet_bc.astype(np.int32), geo=mesh.geo_nodes.astype(np.float64),
                  vx=q.vol_x, vw=q.vol_w, fx=q.fct_x, fw=q.fct_w, c0=c0)
    if c1 is not None:
        arrays["c1"] = c1
    x = np.random.default_rng(seed).standard_normal(op.ndof)
    arrays["x"] = x
    for k, v in arrays.items():
        np.ascontiguousarray(v).tofile(tmp / f"{k}.bin")
    return q, c0, c1, x


def _run(tmp: Path, mode: str) -> dict:
    r = subprocess.run([str(_driver()), str(tmp), mode], capture_output=True, text=True, timeout=300)
    lines = dict(ln.split(" ", 1) for ln in r.stdout.strip().splitlines() if " " in ln)
    assert r.returncode == 0, r.stdout + r.stderr
    return lines


CASES = [("poisson2d", 2, 4, 2, 0), ("elasticity3d", 3, 2, 4, 1)]


@pytest.mark.parametrize("name,dim,n,degree,kind", CASES, ids=[c[0] for c in CASES])
def test_glue_compiles_and_reports_errors(tmp_path, name, dim, n, degree, kind):
    _write_inputs(tmp_path, make_mesh(dim, n, degree, curved=dim == 3), degree, kind)
    out = _run(tmp_path, "cpu")
    for key in ("invalid_topology_throws", "num_local_elements", "apply_before_material_is_petsc_err_lib",
                "apply_before_material_message", "short_vector_is_petsc_err_lib", "flops_apply_positive",
                "null_arrays_invalid"):
        assert out.get(key) == "ok", (key, out)


@pytest.mark.gpu
@pytest.mark.parametrize("name,dim,n,degree,kind", CASES, ids=[c[0] for c in CASES])
def test_glue_matmult_and_pcshell_on_device(tmp_path, name, dim, n, degree, kind):
    from oracle import Oracle
    mesh = mixed_bc_mesh(dim, n, degree, curved=True)
    q, c0, c1, x = _write_inputs(tmp_path, mesh, degree, kind)
    out = _run(tmp_path, "gpu")
    assert out.get("matmult") == "ok" and out.get("pc_bjacobi") == "ok" and out.get("pc_multigrid") == "ok", out
    orc = Oracle(mesh, degree, kind, q)
    orc.set_material(c0, c1)
    y = np.fromfile(tmp_path / "y.bin")
    ref = orc.apply(x)
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()
    z = np.fromfile(tmp_path / "z.bin")
    D = orc.assemble_diag()
    bs = orc.bs
    zr = np.concatenate([np.linalg.solve(D[e], x[e * bs:(e + 1) * bs]) for e in range(orc.E)])
    assert np.abs(z - zr).max() <= 1e-10 * np.abs(zr).max()
    zm = np.fromfile(tmp_path / "zm.bin")
    assert np.all(np.isfinite(zm)) and np.linalg.norm(zm) > 0
