"""ctypes binding of the in-tree C ABI library (``libbeep3_b200.so``).

The library is the product: every compute entry point runs on the GPU.  If
it is missing or cannot be loaded this module raises immediately; there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libbeep3_b200.so"

BP_OK = 0
BP_ERR_INVALID = 1
BP_ERR_CUDA = 2
BP_ERR_NOMEM = 3
BP_ERR_BUDGET = 4
BP_ERR_TIMEOUT = 5
BP_ERR_INTERNAL = 6
BP_ERR_UNSUPPORTED = 7
BP_ERR_NOT_CONVERGED = 8

BP_PREC_FP64 = 0
BP_PREC_MIXED = 1

BP_FLAG_NEARFIELD_ON_DEMAND = 1
BP_FLAG_DEVICE_TREE = 2
BP_FLAG_COMPACT_NEARFIELD = 4
BP_FLAG_MESH_PAIR_CACHE = 8

_ERR_NAMES = {
    BP_ERR_INVALID: "invalid argument", BP_ERR_CUDA: "CUDA error", BP_ERR_NOMEM: "out of host memory",
    BP_ERR_BUDGET: "HBM budget exceeded", BP_ERR_TIMEOUT: "device wait timed out",
    BP_ERR_INTERNAL: "internal error", BP_ERR_UNSUPPORTED: "unsupported", BP_ERR_NOT_CONVERGED: "not converged",
}


class BeepError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{_ERR_NAMES.get(code, code)}: {message}")
        self.code = code


class BudgetExceeded(BeepError):
    pass


class NotConverged(BeepError):
    pass


class bp_patches(C.Structure):
    _fields_ = [
        ("n_patches", C.c_int32),
        ("centroid", C.c_void_p), ("normal", C.c_void_p), ("area", C.c_void_p),
        ("dielectric_ratio", C.c_void_p), ("gc", C.c_void_p),
        ("qual_offsets", C.c_void_p), ("qual_points", C.c_void_p),
        ("quad_offsets", C.c_void_p), ("quad_points", C.c_void_p),
        ("galerkin_offsets", C.c_void_p), ("galerkin_points", C.c_void_p),
    ]


class bp_params(C.Structure):
    _fields_ = [
        ("kappa", C.c_double), ("beta0", C.c_double), ("cube_centre", C.c_double * 3), ("cube_edge", C.c_double),
        ("nbsize", C.c_int32), ("nterms", C.c_int32), ("precision", C.c_int32), ("flags", C.c_int32),
    ]


class bp_instance(C.Structure):
    _fields_ = [
        ("mesh", C.c_void_p), ("rotation", C.c_double * 9), ("offset", C.c_double * 3),
        ("dielectric_ratio", C.c_double),
    ]


class bp_problem_info(C.Structure):
    _fields_ = [
        ("n_patches", C.c_int64), ("n_levels", C.c_int64), ("n_nodes", C.c_int64), ("n_leaves", C.c_int64),
        ("n_nearfield_pairs", C.c_int64), ("n_nearfield_cols", C.c_int64), ("fmm_active", C.c_int64), ("device_bytes", C.c_uint64),
        ("tree_ms", C.c_double), ("assemble_ms", C.c_double), ("gmres_graph", C.c_int64),
        ("fmm_setup_ms", C.c_double), ("setup_ms", C.c_double), ("n_scenarios", C.c_int64),
        ("fmm_m2x_cols", C.c_int64), ("fmm_x2l_cols", C.c_int64), ("fmm_translations", C.c_int64),
        ("fmm_shift_cols", C.c_int64), ("fmm_plane_waves", C.c_int64), ("fmm_coefficients", C.c_int64),
    ]


_P = C.c_void_p
_I = C.c_int32
_D = C.c_double
_PP = C.POINTER(C.c_void_p)

# name -> argtypes; every function returns int32 status unless listed in _RET
_SIGS = {
    "bp_last_error": [],
    "bp_abi_version": [],
    "bp_ctx_create": [_I, C.c_uint64, _PP],
    "bp_ctx_destroy": [_P],
    "bp_ctx_set_stream": [_P, _P],
    "bp_ctx_memory": [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)],
    "bp_ctx_synchronize": [_P],
    "bp_ctx_cache": [_P, C.POINTER(C.c_uint64), _I],
    "bp_geom_create": [_I, _P, _P, _I, _P, _I, _I, _I, _PP],
    "bp_geom_sizes": [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)],
    "bp_geom_copy": [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "bp_geom_destroy": [_P],
    "bp_problem_create": [_P, C.POINTER(bp_patches), C.POINTER(bp_params), _PP],
    "bp_mesh_create": [_P, C.POINTER(bp_patches), _P, _PP],
    "bp_mesh_create_from_surface": [_P, _I, _P, _P, _I, _P, _I, _I, _I, _P, _PP, _P],
    "bp_mesh_destroy": [_P],
    "bp_problem_create_posed": [_P, C.POINTER(bp_instance), _I, C.POINTER(bp_params), _PP],
    "bp_problem_create_batch": [_P, C.POINTER(bp_instance), _I, _P, _I, _P, C.POINTER(bp_params), _PP],
    "bp_problem_destroy": [_P],
    "bp_problem_info_get": [_P, C.POINTER(bp_problem_info)],
    "bp_problem_tree": [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(C.c_int64), _P, _P, _P],
    "bp_tree_create": [_I, _P, _P, _D, _I, _PP],
    "bp_tree_export": [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(C.c_int64), _P, _P, _P],
    "bp_tree_destroy": [_P],
    "bp_matvec": [_P, _P, _P],
    "bp_matvec_device": [_P, _P, _P],
    "bp_matvec_profile": [_P, _P, _P, _I, _P, _P, C.POINTER(_I)],
    "bp_problem_test_wait_timeout": [_P, _I],
    "bp_solve": [_P, _P, _P, _D, _I, _I, C.POINTER(_I), C.POINTER(_D)],
    "bp_solve_device": [_P, _P, _P, _D, _I, _I, C.POINTER(_I), C.POINTER(_D)],
    "bp_solve_batch": [_P, _P, _P, _D, _I, _I, _P, _P],
    "bp_rhs": [_P, _P, _I, _D, _P],
    "bp_rhs_posed": [_P, _P, _P, _D, _P],
    "bp_rhs_noalloc": [_I, _P, _P, _I, _P, _I, _D, _P, _P],
    "bp_energy_coefficients": [_P, _I, _I, _P, _I, _D, _P, _P],
    "bp_energy": [_P, _I, _I, _P, _P, _D, _P, C.POINTER(_D)],
}
_RET = {"bp_last_error": C.c_char_p}

_lib = None


def exported_symbols() -> list[str]:
    return list(_SIGS)


def lib() -> C.CDLL:
    """Loads the library once; raises if it is absent (no fallback)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run `python beep3_b200/build.py` (needs nvcc)")
        L = C.CDLL(str(LIB_PATH))
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RET.get(name, C.c_int32)
        _lib = L
    return _lib


def check(code: int) -> None:
    if code == BP_OK:
        return
    msg = lib().bp_last_error().decode(errors="replace")
    if code == BP_ERR_BUDGET:
        raise BudgetExceeded(code, msg)
    if code == BP_ERR_NOT_CONVERGED:
        raise NotConverged(code, msg)
    raise BeepError(code, msg)


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the C ABI must be contiguous"
    return a.ctypes.data
