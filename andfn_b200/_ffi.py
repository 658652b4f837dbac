"""ctypes binding of libandfn_b200.so (include/andfn_b200.h).

The library must exist in-tree; there is no fallback implementation, so a
missing or unloadable library raises immediately.
"""
from __future__ import annotations

import ctypes
import os

from .records import AndfnAdjointStats, AndfnConstants, AndfnLayout, AndfnResidual, AndfnSolveStats

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libandfn_b200.so")

EXPORTS = ("andfn_b200_solve", "andfn_b200_create", "andfn_b200_upload_state", "andfn_b200_reset_state",
           "andfn_b200_run", "andfn_b200_download", "andfn_b200_eval_heads", "andfn_b200_eval_omega",
           "andfn_b200_destroy", "andfn_b200_stream", "andfn_b200_last_error", "andfn_b200_version",
           "andfn_b200_set_profiling", "andfn_b200_kernel_times", "andfn_b200_fp64_peak",
           "andfn_b200_batch_solve", "andfn_b200_batch_create", "andfn_b200_batch_run",
           "andfn_b200_batch_download", "andfn_b200_batch_eval_heads", "andfn_b200_realizations",
           "andfn_b200_eval_heads_noalloc", "andfn_b200_adjoint", "andfn_b200_set_transmissivity",
           "andfn_b200_state_device", "andfn_b200_heads_device", "andfn_b200_heads_vjp",
           "andfn_b200_bc_residual", "andfn_b200_eval_w", "andfn_b200_eval_w_object",
           "andfn_b200_track", "andfn_b200_disc_intersections", "andfn_b200_clusters",
           "andfn_b200_geometry_last_error", "andfn_b200_release_cached_memory", "andfn_b200_cached_memory")

STATUS = {0: "ok", 1: "max_iterations", 2: "nonfinite", 3: "singular", 10: "bad_layout", 11: "bad_input",
          12: "cuda_error", 13: "no_device", 14: "out_of_memory"}

_lib = None


class AndfnError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"andfn_b200 error {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m andfn_b200.build` "
                          "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    P, I64, I32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32
    LP = ctypes.POINTER(AndfnLayout)
    CP = ctypes.POINTER(AndfnConstants)
    SP = ctypes.POINTER(AndfnSolveStats)
    for name, res, args in (
        ("andfn_b200_solve", ctypes.c_int, [P, I64, P, I64, LP, I64, CP, SP]),
        ("andfn_b200_create", ctypes.c_int, [ctypes.POINTER(P), P, I64, P, I64, LP, I64, I32]),
        ("andfn_b200_upload_state", ctypes.c_int, [P, P, P]),
        ("andfn_b200_reset_state", ctypes.c_int, [P]),
        ("andfn_b200_run", ctypes.c_int, [P, CP, SP]),
        ("andfn_b200_download", ctypes.c_int, [P, P, P]),
        ("andfn_b200_eval_heads", ctypes.c_int, [P, P, P, I64, P]),
        ("andfn_b200_eval_omega", ctypes.c_int, [P, P, P, I64, P]),
        ("andfn_b200_eval_w", ctypes.c_int, [P, P, P, I64, P]),
        ("andfn_b200_eval_w_object", ctypes.c_int, [P, P, P, I64, P]),
        ("andfn_b200_track", ctypes.c_int, [P, P, I64, P, I64, P, P, P, ctypes.c_double, I64, I32, I64,
                                            P, P, P, P, P, P, P]),
        ("andfn_b200_destroy", None, [P]),
        ("andfn_b200_stream", P, [P]),
        ("andfn_b200_last_error", ctypes.c_char_p, []),
        ("andfn_b200_version", ctypes.c_char_p, []),
        ("andfn_b200_set_profiling", ctypes.c_int, [P, ctypes.c_int]),
        ("andfn_b200_kernel_times", ctypes.c_int, [P, P, P, ctypes.c_int]),
        ("andfn_b200_fp64_peak", ctypes.c_int, [I32, P]),
        ("andfn_b200_batch_solve", ctypes.c_int, [I64, P, P, P, P, LP, I64, CP, P]),
        ("andfn_b200_batch_create", ctypes.c_int, [ctypes.POINTER(P), I64, P, P, P, P, LP, I64, I32]),
        ("andfn_b200_batch_run", ctypes.c_int, [P, CP, P]),
        ("andfn_b200_batch_download", ctypes.c_int, [P, P, P]),
        ("andfn_b200_batch_eval_heads", ctypes.c_int, [P, I64, P, P, I64, P]),
        ("andfn_b200_realizations", I64, [P]),
        ("andfn_b200_eval_heads_noalloc", ctypes.c_int, [P, P, P, I64, P]),
        ("andfn_b200_adjoint", ctypes.c_int, [P, P, I64, P, P, ctypes.c_double, I64, P,
                                              ctypes.POINTER(AndfnAdjointStats)]),
        ("andfn_b200_set_transmissivity", ctypes.c_int, [P, P]),
        ("andfn_b200_state_device", ctypes.c_int, [P, P, I64, P, P]),
        ("andfn_b200_heads_device", ctypes.c_int, [P, P, P, I64, P]),
        ("andfn_b200_heads_vjp", ctypes.c_int, [P, P, P, I64, P, P, I64, P, P, P]),
        ("andfn_b200_bc_residual", ctypes.c_int, [P, P, P, ctypes.POINTER(AndfnResidual)]),
        ("andfn_b200_disc_intersections", ctypes.c_int, [I32, I64, P, P, P, P, P, ctypes.c_double, I64, P, P, P,
                                                         P]),
        ("andfn_b200_clusters", ctypes.c_int, [I32, I64, I64, P, P]),
        ("andfn_b200_geometry_last_error", ctypes.c_char_p, []),
        ("andfn_b200_release_cached_memory", None, []),
        ("andfn_b200_cached_memory", ctypes.c_int, [I32, P, P, P]),
    ):
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    return lib().andfn_b200_last_error().decode(errors="replace")


def check(code: int, ok=(0,)):
    if code not in ok:
        raise AndfnError(code, last_error())
    return code
