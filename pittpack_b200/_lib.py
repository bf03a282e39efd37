"""ctypes binding of libpittpack_b200.so (the C ABI in include/pittpack_b200.h).

The product path: if the library is missing, the first call that needs it
raises ImportError with the build command; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpittpack_b200.so")

PP_SUCCESS = 0
PP_INPUT_ARGS = 19
PP_INVALID_HANDLE = 24
PP_NOT_READY = 25
PP_UNSUPPORTED = 27
PP_PRECISION_FP64 = 0
PP_PRECISION_MIXED = 1
PP_ZSOLVE_DIRECT = 0
PP_ZSOLVE_MULTIGRID = 1
PP_ZSOLVE_REF_PCR = 2
PP_ZSOLVE_REF_CRP = 3


class Options(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int),
        ("max_sweeps", ctypes.c_int),
        ("tolerance", ctypes.c_double),
        ("compat_zero_mode", ctypes.c_int),
        ("dirichlet_lift", ctypes.c_int),
        ("z_solver", ctypes.c_int),
        ("zero_mean", ctypes.c_int),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [("zsolve_lanes", ctypes.c_int), ("line_tile", ctypes.c_int), ("zsolve_tile", ctypes.c_int)]


class PittPackError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what}: {result_string(code)} (code {code})")


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m pittpack_b200.build` "
            "(the solver has no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    H = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    i = ctypes.c_int
    sig = {
        "pp_result_string": ([i], ctypes.c_char_p),
        "pp_create": ([i, i, i, ctypes.POINTER(H)], i),
        "pp_destroy": ([H], i),
        "pp_set_box": ([H, dp], i),
        "pp_assign_boundary": ([H, ctypes.c_char_p], i),
        "pp_set_face_values": ([H, i, ctypes.c_void_p], i),
        "pp_default_options": ([ctypes.POINTER(Options)], i),
        "pp_set_options": ([H, ctypes.POINTER(Options)], i),
        "pp_get_options": ([H, ctypes.POINTER(Options)], i),
        "pp_assign_rhs": ([H, ctypes.c_void_p], i),
        "pp_assign_rhs_complex": ([H, ctypes.c_void_p], i),
        "pp_assign_rhs_device": ([H, ctypes.c_void_p, i], i),
        "pp_solve": ([H], i),
        "pp_get_solution": ([H, ctypes.c_void_p], i),
        "pp_profile_solve": ([H, dp, i], i),
        "pp_timing_begin": ([H, i], i),
        "pp_timing_end": ([H, dp, i, ctypes.POINTER(i)], i),
        "pp_get_solution_device": ([H, ctypes.c_void_p], i),
        "pp_solution_device_ptr": ([H, ctypes.POINTER(ctypes.c_void_p)], i),
        "pp_get_error_manufactured": ([H, dp], i),
        "pp_fill_trigonometric": ([H, ctypes.c_void_p], i),
        "pp_fill_trigonometric_box": ([i, i, i, dp, ctypes.c_void_p], i),
        "pp_io": ([ctypes.c_void_p, ctypes.c_uint, i, i], i),
        "pp_set_slab": ([H, i, i], i),
        "pp_stage_forward": ([H], i),
        "pp_stage_spectrum": ([H, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(i), ctypes.POINTER(i)], i),
        "pp_stage_zsolve": ([H, ctypes.c_void_p, i, i, i], i),
        "pp_stage_inverse": ([H], i),
        "pp_zsolve_stats": ([H, ctypes.POINTER(i), ctypes.POINTER(i)], i),
        "pp_set_stream": ([H, ctypes.c_void_p], i),
        "pp_synchronize": ([H], i),
        "pp_host_alloc": ([ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)], i),
        "pp_host_free": ([ctypes.c_void_p], i),
        "pp_workspace_bytes": ([H, ctypes.POINTER(ctypes.c_size_t)], i),
        "pp_assign_rhs_async": ([H, ctypes.c_void_p], i),
        "pp_get_solution_async": ([H, ctypes.c_void_p], i),
        "pp_get_solution_real": ([H, ctypes.c_void_p], i),
        "pp_kernel_timeouts": ([H, ctypes.POINTER(i)], i),
        "pp_get_solution_real_async": ([H, ctypes.c_void_p], i),
        "pp_bind_device_buffers": ([H, ctypes.c_void_p, i, ctypes.c_void_p], i),
        "pp_set_tuning": ([H, ctypes.POINTER(Tuning)], i),
        "pp_get_tuning": ([H, ctypes.POINTER(Tuning)], i),
        "pp_autotune": ([H, i, ctypes.POINTER(Tuning), dp], i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def result_string(code: int) -> str:
    return load().pp_result_string(code).decode()


def check(code: int, what: str) -> None:
    if code != PP_SUCCESS:
        raise PittPackError(code, what)
