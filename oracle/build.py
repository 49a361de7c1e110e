"""ORACLE -- test infrastructure only.  Build recipe of the CPU oracle.

* ``oracle/_build/liboracle.so``: the C++ restatement (oracle.cpp) with the reference-element
  tables of the product (``tandem_b200/csrc/host/refelem.cpp``), g++ -O3 -march=native -fopenmp.
* ``oracle/_ref/libtandem_ref.so``: tandem's own Eigen-free quadrature and basis sources compiled
  in place from the reference tree (src/quadrules/*.cpp, src/basis/Functions.cpp,
  src/util/Math.cpp) with the C shim ``ref_shim.cpp``; built only where the reference tree is
  present (its output travels with the repository snapshot, the sources do not).
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
BUILD = HERE / "_build"
REF_OUT = HERE / "_ref"
LIB = BUILD / "liboracle.so"
REF_LIB = REF_OUT / "libtandem_ref.so"
REFERENCE = Path(os.environ.get("TANDEM_REFERENCE", "/root/reference"))

REF_SOURCES = ["src/quadrules/GaussJacobi.cpp", "src/quadrules/IntervalQuadratureRule.cpp",
               "src/quadrules/TensorProductRule.cpp", "src/quadrules/JaskowiecSukumar2020.cpp",
               "src/quadrules/WitherdenVincent2015_Tri.cpp", "src/quadrules/WitherdenVincent2015_Tet.cpp",
               "src/basis/Functions.cpp", "src/util/Math.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")


def build_oracle(force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = [HERE / "oracle.cpp", ROOT / "tandem_b200/csrc/host/refelem.cpp"]
    deps = srcs + [ROOT / "tandem_b200/csrc/host/refelem.hpp", ROOT / "include/tandem_b200.h"]
    if force or not LIB.exists() or any(LIB.stat().st_mtime < p.stat().st_mtime for p in deps):
        _run(["g++", "-O3", "-march=native", "-fopenmp", "-std=c++17", "-fPIC", "-shared",
              "-o", str(LIB), *map(str, srcs)])
    return LIB


def build_reference(force: bool = False) -> Path | None:
    """Compiles tandem's quadrature/basis sources where they lie; None if the tree is absent."""
    if not (REFERENCE / "src/quadrules/AutoRule.h").exists():
        return REF_LIB if REF_LIB.exists() else None
    REF_OUT.mkdir(exist_ok=True)
    if force or not REF_LIB.exists():
        srcs = [str(REFERENCE / s) for s in REF_SOURCES]
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", str(REFERENCE / "src"),
              "-o", str(REF_LIB), str(HERE / "ref_shim.cpp"), *srcs])
    return REF_LIB


def build(force: bool = False) -> None:
    build_oracle(force)
    build_reference(force)


if __name__ == "__main__":
    build(force=True)
    print(LIB, REF_LIB if REF_LIB.exists() else "(reference tree absent)")
