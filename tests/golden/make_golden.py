"""Generates the golden fixtures under tests/golden/ from the reference tree.

* ``quadrature.json``: tandem's simplexQuadratureRule<D>(order) (AutoRule: Witherden-Vincent /
  Jaskowiec-Sukumar tables, Gauss-Jacobi conical rules) and TensorProductRule<D>::get(order),
  evaluated by tandem's own sources compiled in place (oracle/_ref).
* ``dubiner.json``: tandem's DubinerP / gradDubinerP / JacobiP / GaussJacobi values.
* ``kat.json``: known-answer values transcribed from tandem's unit tests: warp & blend and
  equidistant nodes (test/basis.cpp:209-420), Gauss-Jacobi vs Maple and the conical triangle rule
  (test/quadrules.cpp:23-50), modal tetrahedron mass matrix (test/form.cpp:19-58), and the AutoRule
  sizes (test/quadrules.cpp:121-133).

Run from the repository root where the reference tree is mounted:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from oracle import build as obuild  # noqa: E402

OUT = Path(__file__).resolve().parent
REF = obuild.REFERENCE


def rules():
    L = oracle.ref_lib()
    out = {"auto": {}, "conical": {}}
    for dim in (1, 2, 3):
        for order in (1, 3, 5, 7, 9, 11):
            for key, fn in (("auto", L.ref_simplex_rule), ("conical", L.ref_conical_rule)):
                n = fn(dim, order, None, None)
                x = np.zeros((n, dim))
                w = np.zeros(n)
                fn(dim, order, x.ctypes.data, w.ctypes.data)
                out[key][f"{dim}:{order}"] = {"points": x.tolist(), "weights": w.tolist()}
    return out


def dubiner():
    L = oracle.ref_lib()
    rng = np.random.default_rng(1234)
    out = {"tri": [], "tet": [], "jacobi": [], "gauss_jacobi": []}
    import ctypes as C
    for dim, key in ((2, "tri"), (3, "tet")):
        pts = rng.dirichlet(np.ones(dim + 1), size=12)[:, :dim]
        for N in range(0, 5):
            for j in _multi(dim, N):
                for p in pts:
                    ja = (C.c_uint * 3)(*(list(j) + [0] * (3 - dim)))
                    xa = (C.c_double * 3)(*(list(p) + [0.0] * (3 - dim)))
                    g = (C.c_double * 3)()
                    v = L.ref_dubiner(dim, ja, xa)
                    L.ref_grad_dubiner(dim, ja, xa, g)
                    out[key].append({"j": list(j), "x": list(map(float, p)), "v": v, "g": list(g)[:dim]})
    for n in range(0, 7):
        for a in range(0, 4):
            for b in range(0, 3):
                for x in (-0.9, -0.3, 0.0, 0.4, 0.95):
                    out["jacobi"].append({"n": n, "a": a, "b": b, "x": x, "v": L.ref_jacobi(n, a, b, x)})
    for n, a, b in ((5, 1, 3), (5, 0, 0), (7, 1, 0), (6, 2, 0), (4, 1, 1)):
        x = np.zeros(n)
        w = np.zeros(n)
        L.ref_gauss_jacobi(n, a, b, x.ctypes.data, w.ctypes.data)
        out["gauss_jacobi"].append({"n": n, "a": a, "b": b, "x": x.tolist(), "w": w.tolist()})
    return out


def _multi(dim, N):
    if dim == 2:
        return [(i, N - i) for i in range(N + 1)]
    return [(i, j, N - i - j) for i in range(N + 1) for j in range(N + 1 - i)]


def _subcase(text: str, name: str) -> str:
    i = text.index(f'SUBCASE("{name}")')
    j = text.index("SUBCASE(", i + 10) if "SUBCASE(" in text[i + 10:] else len(text)
    return text[i:j]


def _numbers(block: str):
    return [float(x) for x in re.findall(r"-?\d+\.\d+(?:[eE][-+]?\d+)?|-?\d+\.(?=\D)|(?<![\w.])-?\d+(?![\w.])", block)]


def _points(block: str, dim: int):
    """Innermost {a, b[, c]} groups of a C++ initializer; entries are literals or quotients."""
    pts = []
    for grp in re.findall(r"\{([^{}]*)\}", block):
        items = [t.strip() for t in grp.split(",") if t.strip()]
        if len(items) != dim or not all(re.fullmatch(r"[-0-9.\s/]+", t) for t in items):
            continue
        vals = []
        for t in items:
            num, *den = [float(u) for u in t.split("/")]
            vals.append(num / den[0] if den else num)
        pts.append(vals)
    return pts


def kat():
    basis = (REF / "test/basis.cpp").read_text()
    out = {"warp_blend": {}, "equidistant": {}}
    for dim, shape in ((2, "Triangle"), (3, "Tet")):
        for N in range(0, 5):
            blk = _subcase(basis, f"{shape} nodes P{N}")
            blk = blk[blk.index("{"):blk.index("checkNodes")]
            if N == 0:
                out["warp_blend"][f"{dim}:{N}"] = [[1.0 / (dim + 1)] * dim]
                continue
            out["warp_blend"][f"{dim}:{N}"] = _points(blk, dim)
    for dim, shape in ((2, "Triangle"), (3, "Tet")):
        for N in (1, 2, 3, 6):
            name = f"{shape} nodes P{N} (equidistant)"
            if f'SUBCASE("{name}")' not in basis:
                continue
            blk = _subcase(basis, name)
            blk = blk[blk.index("{"):blk.index("checkNodes")]
            out["equidistant"][f"{dim}:{N}"] = _points(blk, dim)
    quad = (REF / "test/quadrules.cpp").read_text()
    gj = _subcase(quad, "Gauss Jacobi vs Maple")
    v = [float(x) for x in re.findall(r"Approx\((-?\d*\.\d+)\)", gj)]
    out["gauss_jacobi_5_1_3"] = {"x": v[:5], "w": v[5:10]}
    tri = _subcase(quad, "Triangle vs Maple")
    v = [float(x) for x in re.findall(r"Approx\((-?\d*\.\d+)\)", tri)]
    out["conical_tri_order3"] = {"x0": v[0:4], "x1": v[4:8], "w": v[8:12]}
    auto = _subcase(quad, "Autorule")
    out["autorule_sizes"] = [[int(a), int(b), int(c)] for a, b, c in
                             re.findall(r"simplexQuadratureRule<(\d)u>\((\d+)\)\.size\(\) == (\d+)", auto)]
    form = (REF / "test/form.cpp").read_text()
    blk = form[form.index("refModalMassMatrix = {"):form.index("};", form.index("refModalMassMatrix = {"))]
    out["modal_mass_tet"] = [float(x) for x in re.findall(r"\.\d+(?:e-?\d+)?", blk)]
    return out


def main():
    obuild.build()
    (OUT / "quadrature.json").write_text(json.dumps(rules()))
    (OUT / "dubiner.json").write_text(json.dumps(dubiner()))
    (OUT / "kat.json").write_text(json.dumps(kat(), indent=1))
    print("wrote", *(p.name for p in OUT.glob("*.json")))


if __name__ == "__main__":
    main()
