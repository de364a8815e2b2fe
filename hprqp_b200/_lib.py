"""ctypes loader for libhprqp.so (the C ABI of include/hprqp.h).

The library is loaded from this package directory.  There is no fallback:
if it is missing or CUDA is unusable, calls raise (the reference silently
fell back to its CPU path, src/utils.jl:14-31; this build does not).
"""
from __future__ import annotations

import ctypes as C
import os

from ._abi import Params, PassStats, Result

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhprqp.so")

# Every entry point declared in include/hprqp.h
EXPORTS = ("hprqp_abi_info", "hprqp_default_params", "hprqp_create", "hprqp_load", "hprqp_prepare",
           "hprqp_solve", "hprqp_set_save_file", "hprqp_solve_resume", "hprqp_set_trace", "hprqp_set_trace_scalars", "hprqp_set_qmap", "hprqp_profile_iterations", "hprqp_get_pass_stats",
           "hprqp_power_lambda_noalloc", "hprqp_gemm_3xtf32", "hprqp_gemm_3xtf32_ws_floats",
           "hprqp_gemm_3xtf32_ws", "hprqp_last_error", "hprqp_destroy")

_lib = None


class HPRQPError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libhprqp error {code}: {msg}")
        self.code = code


def load():
    """Load libhprqp.so (build it first with hprqp_b200.build if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise HPRQPError(-4, f"{LIB_PATH} not built; run `python -m hprqp_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.hprqp_abi_info.argtypes = [C.POINTER(C.c_int64)]
    L.hprqp_abi_info.restype = C.c_int
    L.hprqp_default_params.argtypes = [C.POINTER(Params)]
    L.hprqp_default_params.restype = None
    L.hprqp_create.argtypes = [C.POINTER(vp), C.c_int32]
    L.hprqp_create.restype = C.c_int
    L.hprqp_load.argtypes = [vp, vp]
    L.hprqp_load.restype = C.c_int
    L.hprqp_prepare.argtypes = [vp, C.POINTER(Params)]
    L.hprqp_prepare.restype = C.c_int
    L.hprqp_solve.argtypes = [vp, C.POINTER(Params), vp, vp, C.POINTER(Result), vp, vp, vp, vp]
    L.hprqp_solve.restype = C.c_int
    L.hprqp_set_trace.argtypes = [vp, C.c_int64, vp, vp, vp]
    L.hprqp_set_trace.restype = C.c_int
    L.hprqp_set_save_file.argtypes = [vp, C.c_char_p]
    L.hprqp_set_save_file.restype = C.c_int
    L.hprqp_solve_resume.argtypes = [vp, C.POINTER(Params), C.c_char_p, C.POINTER(Result), vp, vp, vp, vp]
    L.hprqp_solve_resume.restype = C.c_int
    L.hprqp_set_trace_scalars.argtypes = [vp, vp, vp]
    from ._abi import QMAP_FN
    L.hprqp_set_qmap.argtypes = [vp, QMAP_FN, vp]
    L.hprqp_set_qmap.restype = C.c_int
    L.hprqp_set_trace_scalars.restype = C.c_int
    L.hprqp_profile_iterations.argtypes = [vp, C.POINTER(Params), C.c_int64, C.c_int32, C.POINTER(PassStats)]
    L.hprqp_profile_iterations.restype = C.c_int
    L.hprqp_get_pass_stats.argtypes = [vp, C.POINTER(PassStats), C.POINTER(PassStats)]
    L.hprqp_get_pass_stats.restype = C.c_int
    L.hprqp_power_lambda_noalloc.argtypes = [C.c_int64, C.c_int64, vp, vp, vp, vp, vp, vp, C.c_int32,
                                             C.c_double, C.c_int32, vp, C.POINTER(C.c_double),
                                             C.POINTER(C.c_int32)]
    L.hprqp_power_lambda_noalloc.restype = C.c_int
    L.hprqp_gemm_3xtf32.argtypes = [C.c_int32, C.c_float, vp, vp, C.c_float, vp, vp]
    L.hprqp_gemm_3xtf32.restype = C.c_int
    L.hprqp_gemm_3xtf32_ws_floats.argtypes = [C.c_int32]
    L.hprqp_gemm_3xtf32_ws_floats.restype = C.c_int64
    L.hprqp_gemm_3xtf32_ws.argtypes = [C.c_int32, C.c_float, vp, vp, C.c_float, vp, vp, vp]
    L.hprqp_gemm_3xtf32_ws.restype = C.c_int
    L.hprqp_last_error.argtypes = [vp]
    L.hprqp_last_error.restype = C.c_char_p
    L.hprqp_destroy.argtypes = [vp]
    L.hprqp_destroy.restype = C.c_int
    _lib = L
    return L


def check(rc, handle=None):
    if rc != 0:
        msg = load().hprqp_last_error(handle).decode(errors="replace")
        raise HPRQPError(rc, msg)
