"""ctypes bindings of the C ABI in ``include/tandem_b200.h``.

The native library is mandatory: importing this module raises if it has not been built; there is
no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libtandem_b200.so"

TDG_POISSON, TDG_ELASTICITY = 0, 1
TDG_BC_NONE, TDG_BC_NATURAL, TDG_BC_FAULT, TDG_BC_DIRICHLET = 0, 1, 3, 5
TDG_FP64, TDG_FP32, TDG_MIXED, TDG_TF32 = 0, 1, 2, 3
ERRORS = {-1: "TDG_E_INVALID", -2: "TDG_E_CUDA", -3: "TDG_E_NOT_SPD", -4: "TDG_E_DIVERGED",
          -5: "TDG_E_STATE", -6: "TDG_E_TIMEOUT", -7: "TDG_E_NOMEM"}
ERRORS_BY_NAME = {v: k for k, v in ERRORS.items()}

# Every symbol the header declares, with (restype, argtypes).
_p = C.c_void_p
_i64 = C.c_int64
SYMBOLS = {
    "tdg_create": (C.c_int, [_p, _p, C.c_int, C.POINTER(_p)]),
    "tdg_destroy": (None, [_p]),
    "tdg_last_error": (C.c_char_p, []),
    "tdg_sizes": (C.c_int, [_p, _p]),
    "tdg_volume_coords": (C.c_int, [_p, _p]),
    "tdg_facet_coords": (C.c_int, [_p, _p]),
    "tdg_facet_normals": (C.c_int, [_p, _p]),
    "tdg_set_material": (C.c_int, [_p, _p, _p]),
    "tdg_update_material": (C.c_int, [_p, _p, _p]),
    "tdg_material_nodal": (C.c_int, [_p, C.c_int, _p]),
    "tdg_penalty": (C.c_int, [_p, _p]),
    "tdg_apply": (C.c_int, [_p, C.c_int, _p, _p, C.c_int, _i64, _p]),
    "tdg_apply_host": (C.c_int, [_p, C.c_int, _p, _p, C.c_int, C.c_int64, _p]),
    "tdg_flops_apply": (_i64, [_p]),
    "tdg_bytes_apply": (_i64, [_p, C.c_int]),
    "tdg_bjacobi_setup": (C.c_int, [_p, C.c_int, _p]),
    "tdg_bjacobi_apply": (C.c_int, [_p, C.c_int, _p, _p, C.c_int, _i64, _p]),
    "tdg_bjacobi_blocks": (C.c_int, [_p, _p]),
    "tdg_rhs": (C.c_int, [_p, _p, _p, _p]),
    "tdg_solve": (C.c_int, [_p, _p, _p, C.c_int, _i64, _p, _p, _p]),
    "tdg_solve_segmented": (C.c_int, [_p, _p, _p, C.c_int, _p, _p, _p, _p, _p]),
    "tdg_solve_distributed": (C.c_int, [_p, _p, _p, _i64, _p, _p, _p, _p, _p, _p]),
    "tdg_adjoint_lame_gradient": (C.c_int, [_p, _p, _p, _p, _p, _p]),
    "tdg_adjoint_lame_gradient_noalloc": (C.c_int, [_p, _p, _p, _p, _p, _p]),
    "tdg_autotune": (C.c_int, [_p, C.c_int, C.c_int, _p, _p, C.c_int, _p]),
    "tdg_set_apply_config": (C.c_int, [_p, C.c_int, C.c_int, C.c_int]),
    "tdg_set_apply_tile": (C.c_int, [_p, C.c_int, C.c_int]),
    "tdg_probe_fp64_peak": (C.c_int, [C.c_int, C.c_int, _p, C.POINTER(C.c_double)]),
    "tdg_probe_tc05_gemm": (C.c_int, [_p, _p, _p, C.c_int, C.c_int, C.c_int, _p]),
    "tdg_probe_tc05_layout": (C.c_int, [_p, _p, _p, C.c_int, C.c_int, C.c_int, _p]),
    "tdg_set_density": (C.c_int, [_p, _p]),
    "tdg_apply_inverse_mass": (C.c_int, [_p, _p, _p, C.c_int, _i64, _p]),
    "tdg_wave_rhs": (C.c_int, [_p, _p, _p, _p, C.c_int, _i64, _p]),
    "tdg_mg_setup": (C.c_int, [_p, _p, _p]),
    "tdg_mg_apply": (C.c_int, [_p, _p, _p, C.c_int, _i64, _p]),
    "tdg_set_preconditioner": (C.c_int, [_p, C.c_int]),
    "tdg_mg_info": (C.c_int, [_p, _p, C.c_int, _p, _p, _p, _p]),
    "tdg_mg_level_matrix": (C.c_int, [_p, C.c_int, _p, _p]),
    "tdg_mg_level_degrees": (C.c_int, [C.c_int, C.c_int, C.c_int, _p]),
    "tdg_mg_interpolation": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _p]),
    "tdg_mg_colouring": (C.c_int, [_p, _p, _p]),
    "tdg_mg_p1_embedding": (C.c_int, [C.c_int, C.c_int, C.c_int, _p]),
    "tdg_rule_coords": (C.c_int, [_p, C.c_int, _p, _p]),
    "tdg_project": (C.c_int, [_p, _p, _p]),
    "tdg_evaluate": (C.c_int, [_p, _p, C.c_int, _p, _p]),
    "tdg_error_l2": (C.c_int, [_p, _p, C.c_int, _p, _p, _p, _p]),
    "tdg_error_h1_semi": (C.c_int, [_p, _p, C.c_int, _p, _p, _p, _p]),
    "tdg_mg_vertex_numbering": (C.c_int, [_p, _p, _p]),
    "tdg_gf_traction_update": (C.c_int, [_i64, _i64, _p, _i64, _p, _i64, C.c_int, _p, C.c_double, _p, _i64, _p]),
    "tdg_fault_create": (C.c_int, [_p, _i64, _p, _p, C.POINTER(_p)]),
    "tdg_fault_destroy": (None, [_p]),
    "tdg_fault_sizes": (C.c_int, [_p, _p]),
    "tdg_fault_slip_rhs": (C.c_int, [_p, _p, _i64, _p, C.c_int, _i64, _p]),
    "tdg_fault_traction": (C.c_int, [_p, _p, _i64, _p, _i64, _p, _i64, C.c_int, _p]),
    "tdg_ref_nodes": (C.c_int, [C.c_int, C.c_int, C.c_int, _p]),
    "tdg_ref_basis": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _p, _p, _p]),
    "tdg_conical_rule": (C.c_int, [C.c_int, C.c_int, _p, _p]),
}


# callbacks of tdg_solve_distributed: exchange(ctx, v, stream), allreduce(ctx, values, count, stream)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p)


class MeshDesc(C.Structure):
    _fields_ = [("dim", C.c_int32), ("degree", C.c_int32), ("geo_degree", C.c_int32),
                ("reserved", C.c_int32), ("num_elements", C.c_int64), ("num_facets", C.c_int64),
                ("geo_nodes", _p), ("facet_up", _p), ("facet_local_no", _p), ("facet_bc", _p)]


class Quadrature(C.Structure):
    _fields_ = [("num_vol_points", C.c_int32), ("num_fct_points", C.c_int32),
                ("vol_points", _p), ("vol_weights", _p), ("fct_points", _p), ("fct_weights", _p)]


class TuneEntry(C.Structure):
    _fields_ = [("family", C.c_int), ("ctas_per_sm", C.c_int), ("tile", C.c_int), ("ms", C.c_double)]


class SolveOpts(C.Structure):
    _fields_ = [("precision", C.c_int32), ("max_iterations", C.c_int32), ("rtol", C.c_double),
                ("inner_rtol", C.c_double), ("max_outer", C.c_int32), ("use_graphs", C.c_int32),
                ("method", C.c_int32), ("restart", C.c_int32)]


TDG_KSP_CG, TDG_KSP_FGMRES = 0, 1


TDG_PC_BJACOBI, TDG_PC_MG = 0, 1
TDG_MG_TWOLEVEL, TDG_MG_LOGARITHMIC, TDG_MG_FULL = 0, 1, 2


class MgOpts(C.Structure):
    _fields_ = [("strategy", C.c_int32), ("coarse_degree", C.c_int32), ("smooth_its", C.c_int32),
                ("esteig_lo", C.c_double), ("esteig_hi", C.c_double), ("esteig_steps", C.c_int32),
                ("coarse_rtol", C.c_double), ("coarse_max_it", C.c_int32), ("smooth_precision", C.c_int32),
                ("coarse_space", C.c_int32)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("outer", C.c_int32), ("rel_residual", C.c_double),
                ("seconds", C.c_double), ("converged", C.c_int32), ("fp64_iterations", C.c_int32)]


class TdgError(RuntimeError):
    pass


_lib = None


def lib() -> C.CDLL:
    """Loads the native library (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"tandem_b200 native library not built: {LIB_PATH} "
                              "(run python -m tandem_b200.build)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SYMBOLS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != 0:
        msg = lib().tdg_last_error().decode(errors="replace")
        raise TdgError(f"{ERRORS.get(rc, rc)}: {msg}")
