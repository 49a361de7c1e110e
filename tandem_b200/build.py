"""Build recipe of the native library ``tandem_b200/_lib/libtandem_b200.so``.

Compiles the host set-up code (C++17, OpenMP) and the CUDA kernels for sm_100a with nvcc,
in-tree, one object per source, then links a shared library exporting the C ABI declared in
``include/tandem_b200.h``.  Run ``python -m tandem_b200.build`` (or ``build()``).
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "_lib"
LIB = OUT / "libtandem_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp,-O3",
              "--expt-relaxed-constexpr", "-I", str(ROOT / "include")]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-march=x86-64-v3", "-I", str(ROOT / "include")]

SOURCES_CU = ["capi.cu", "kernels/apply.cu", "kernels/bjacobi.cu", "kernels/fault.cu", "kernels/adjoint.cu", "kernels/apply_tc32.cu", "kernels/apply_face.cu", "kernels/apply_face_tc32.cu", "kernels/wave.cu", "kernels/mg.cu", "kernels/peak.cu", "kernels/gf_traction.cu", "kernels/apply_face2.cu", "kernels/tc05_probe.cu", "kernels/apply_tc05.cu"]
SOURCES_CXX = ["host/refelem.cpp", "host/setup.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers_digest() -> str:
    h = hashlib.sha256()
    for p in sorted(list(CSRC.rglob("*.cuh")) + list(CSRC.rglob("*.hpp")) + [ROOT / "include" / "tandem_b200.h"]):
        h.update(p.read_bytes())
    return h.hexdigest()[:16]


def _compile(src: Path, obj: Path, cmd: list[str]) -> str:
    obj.parent.mkdir(parents=True, exist_ok=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src}\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(verbose: bool = False, force: bool = False) -> Path:
    nvcc = _nvcc()
    OUT.mkdir(parents=True, exist_ok=True)
    objdir = OUT / "obj"
    digest = _headers_digest()
    stamp = objdir / "headers.sha"
    if stamp.exists() and stamp.read_text() != digest:
        force = True
    jobs = []
    for s in SOURCES_CU:
        src = CSRC / s
        obj = objdir / (s.replace("/", "_") + ".o")
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-Xptxas", "-v" if verbose else "-O3", "-c", str(src), "-o", str(obj)]
        jobs.append((src, obj, cmd))
    for s in SOURCES_CXX:
        src = CSRC / s
        obj = objdir / (s.replace("/", "_") + ".o")
        cmd = ["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
        jobs.append((src, obj, cmd))
    todo = [j for j in jobs if force or not j[1].exists() or j[1].stat().st_mtime < j[0].stat().st_mtime]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            futs = {ex.submit(_compile, *j): j for j in todo}
            for f in cf.as_completed(futs):
                log = f.result()
                if verbose and log:
                    print(log, file=sys.stderr)
    objs = [str(j[1]) for j in jobs]
    if todo or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc, *ARCH, "-shared", "-Xcompiler", "-fopenmp", "-o", str(tmp), *objs, "-lcudart", "-lgomp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    stamp.write_text(digest)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
