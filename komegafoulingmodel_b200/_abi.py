"""ctypes declarations of the C ABI in include/kofm.h (libkofm.so).

The library is built in-tree for sm_100a (komegafoulingmodel_b200/build.py).
There is no CPU fallback: if the library or a B200 is missing, the calls
raise.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# KOFM_LIBRARY selects another build of the same ABI (e.g. a differently
# configured libkofm.so); the default is the in-tree build.
LIB_PATH = os.environ.get("KOFM_LIBRARY") or os.path.join(HERE, "libkofm.so")

KOFM_OK = 0
ERRORS = {
    -101: "BUFFER_ALLOCATION", -103: "MEMORY_COPY", -107: "CALLING_KERNEL",
    -110: "LOADING_PARAMS", -111: "INITIALIZING_KOMEGA", -112: "INITIALIZING_VLS",
    -120: "INITIALIZING_VLB", -200: "INVALID_ARG", -201: "NO_DEVICE",
    -202: "NOT_CONVERGED", -203: "NAN", -204: "TIMEOUT", -205: "STATE",
    -206: "TOO_LARGE",
}
ERR_INVALID_ARG = -200
ERR_STATE = -205
ERR_TOO_LARGE = -206
NOALLOC_MAX_NODES = 4096 * 65536
ERR_NOT_CONVERGED = -202
ERR_NAN = -203
ERR_TIMEOUT = -204

OPTION_SAVE_MACRO_FIELDS = 0x2
STORE_FP32, STORE_FP16_DEV, STORE_BF16_DEV, STORE_FP16_NEQ, STORE_FP64, STORE_FP16_NEQ32 = 0, 1, 2, 3, 4, 5
STORE_FP16_ROW = 6
FIELD_RHO, FIELD_UX, FIELD_UY, FIELD_K, FIELD_OMEGA, FIELD_NUT, FIELD_WALL_SHEAR, FIELD_TEMP = range(8)
WALLS_IBB_ALL, WALLS_SEAM_IBB = 1, 2
OP_SUM, OP_MIN, OP_MAX = 0, 1, 2


class KofmDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("nx_full", C.c_int32), ("ny", C.c_int32),
        ("use_komega", C.c_int32),
        ("tau", C.c_double), ("fterm", C.c_double), ("mu", C.c_double),
        ("max_turb_visc", C.c_double),
        ("storage", C.c_int32), ("device", C.c_int32),
        ("komega_max_iters", C.c_int32), ("krylov_dim", C.c_int32),
        ("komega_rel_tol", C.c_double), ("komega_abs_tol", C.c_double),
        ("komega_dt", C.c_double),
        ("komega_full_cycle", C.c_int32),
        ("solver_max_blocks", C.c_int32),
        ("use_thermal", C.c_int32), ("thermal_every", C.c_int32),
        ("pr_number", C.c_double), ("pr_turb_number", C.c_double),
        ("alpha_foul", C.c_double), ("t_in", C.c_double),
        ("thermal_max_iters", C.c_int32), ("komega_classic", C.c_int32),
        ("thermal_rel_tol", C.c_double), ("thermal_abs_tol", C.c_double),
        ("thermal_dt", C.c_double),
    ]


class KofmStats(C.Structure):
    _fields_ = [
        ("omega_iters", C.c_int32), ("k_iters", C.c_int32),
        ("omega_restarts", C.c_int32), ("k_restarts", C.c_int32),
        ("omega_cycles", C.c_int32), ("k_cycles", C.c_int32),
        ("omega_vectors", C.c_int32), ("k_vectors", C.c_int32),
        ("omega_vec_index_sum", C.c_int32), ("k_vec_index_sum", C.c_int32),
        ("omega_update_terms", C.c_int32), ("k_update_terms", C.c_int32),
        ("omega_nan", C.c_int32), ("k_nan", C.c_int32),
        ("steps_per_lb", C.c_int32), ("time_since_change", C.c_int32),
        ("dt", C.c_double), ("omega_rel_res", C.c_double), ("k_rel_res", C.c_double),
        ("steps", C.c_int64), ("solver_passes", C.c_int32), ("phase", C.c_int32),
        ("thermal_iters", C.c_int32), ("thermal_checks", C.c_int32),
        ("thermal_solves", C.c_int32), ("thermal_resets", C.c_int32),
        ("thermal_steps_per_lb", C.c_int32), ("thermal_time_since_change", C.c_int32),
        ("thermal_dt", C.c_double), ("thermal_residual", C.c_double),
        ("solver_bytes_per_node", C.c_double), ("omega_powers", C.c_int32), ("k_powers", C.c_int32),
        ("solver_launches", C.c_int32), ("solver_rounds", C.c_int32),
        ("solver_launches_total", C.c_int64),
    ]


# name -> (restype, argtypes)
_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_i16p = C.POINTER(C.c_int16)
_i32p = C.POINTER(C.c_int32)
SIGNATURES = {
    "kofm_abi_version": (C.c_int, []),
    "kofm_error_string": (C.c_char_p, [C.c_int]),
    "kofm_desc_default": (C.c_int, [C.POINTER(KofmDesc)]),
    "kofm_create": (C.c_int, [C.POINTER(KofmDesc), C.POINTER(_vp)]),
    "kofm_destroy": (C.c_int, [_vp]),
    "kofm_set_geometry": (C.c_int, [_vp, _i16p, _dp, _dp, _i32p, _dp, C.c_int32]),
    "kofm_set_walls": (C.c_int, [_vp, _dp, _dp, _dp, _dp, C.c_double, C.c_int32, C.c_int32]),
    "kofm_get_geometry": (C.c_int, [_vp, _i16p, _dp, _dp, _dp, _i32p, _dp, C.c_int32, _i32p]),
    "kofm_set_state": (C.c_int, [_vp, _dp, _dp, _dp, _dp, _dp]),
    "kofm_get_state": (C.c_int, [_vp, _dp, _dp, _dp, _dp, _dp]),
    "kofm_get_macro": (C.c_int, [_vp, _dp, _dp, _dp]),
    "kofm_lb_step": (C.c_int, [_vp, C.c_int32]),
    "kofm_komega_assemble": (C.c_int, [_vp, C.c_double]),
    "kofm_komega_solve": (C.c_int, [_vp, _i32p, _dp]),
    "kofm_komega_update": (C.c_int, [_vp]),
    "kofm_step": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "kofm_reduce": (C.c_int, [_vp, C.c_int32, C.c_int32, _dp]),
    "kofm_sync": (C.c_int, [_vp]),
    "kofm_set_shear": (C.c_int, [_vp, _i32p, C.c_int32, _dp, _i32p, _dp, C.c_int32]),
    "kofm_wall_shear": (C.c_int, [_vp, _dp, _dp]),
    "kofm_get_stats": (C.c_int, [_vp, C.POINTER(KofmStats)]),
    "kofm_debug_barrier_timeout": (C.c_int, [_vp, C.c_int64]),
    "kofm_debug_fail_solves": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "kofm_debug_solver_trace": (C.c_int, [_vp, C.POINTER(C.c_int64), C.c_int32, _i32p]),
    "kofm_debug_komega_rows": (C.c_int, [_vp, C.c_int32, _dp, _dp]),
    "kofm_stream": (_vp, [_vp]),
    "kofm_reduce_field_noalloc": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                            _vp, _vp]),
    "kofm_batch_create": (C.c_int, [C.POINTER(_vp), C.c_int32, C.POINTER(_vp)]),
    "kofm_batch_create_tiled": (C.c_int, [C.POINTER(_vp), C.c_int32, C.c_int32, C.POINTER(_vp)]),
    "kofm_batch_step": (C.c_int, [_vp, C.c_int32]),
    "kofm_batch_destroy": (C.c_int, [_vp]),
    "kofm_set_temperature": (C.c_int, [_vp, _dp]),
    "kofm_get_temperature": (C.c_int, [_vp, _dp]),
    "kofm_set_thermal_geometry": (C.c_int, [_vp, _dp]),
    "kofm_thermal_update": (C.c_int, [_vp]),
    "kofm_adjoint": (C.c_int, [_vp, C.c_int32, _dp, _dp]),
    "kofm_set_adjoint_memory": (C.c_int, [_vp, C.c_int64]),
}

_LIB = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Loads libkofm.so and declares every ABI symbol (raises if absent)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} not built: run `python -m komegafoulingmodel_b200.build` "
            "(nvcc, sm_100a); there is no CPU fallback")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


class KofmError(RuntimeError):
    def __init__(self, fn: str, status: int):
        self.status = status
        super().__init__(f"{fn} -> {status} ({ERRORS.get(status, 'unknown')})")


def check(fn: str, status: int) -> int:
    if status != KOFM_OK:
        raise KofmError(fn, status)
    return status
