"""ctypes binding of libmarfa_gpu.so (C ABI declared in include/marfa_gpu.h).

The library is loaded from the package folder; a missing library is an error
(there is no CPU fallback).
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmarfa_gpu.so"

MARFA_NT = 20481
SHAPE = {"voigt": 0, "lorentz": 1, "one": 100, "absx": 101}
CHI = {"none": 0, "tonkov": 1, "pollack": 2, "perrin": 3}
TARGET = {"ACS": 0, "VAC": 1}
PRECISION = {"fp64": 0, "fp32c": 1}

# every entry point declared in include/marfa_gpu.h
EXPORTS = (
    "marfa_ctx_create", "marfa_ctx_destroy", "marfa_last_error", "marfa_num_subintervals",
    "marfa_record_number", "marfa_compute", "marfa_compute_batched", "marfa_compute_device",
    "marfa_synchronize", "marfa_eval_count", "marfa_debug_accumulators", "marfa_last_timings",
    "marfa_plan_windows", "marfa_compute_record_static", "marfa_ctx_set_tips_grid",
    "marfa_ctx_set_line_params", "marfa_vjp", "marfa_graph_create", "marfa_graph_launch",
    "marfa_graph_destroy", "marfa_autotune", "marfa_ctx_set_launch", "marfa_ctx_get_launch",
)


class MarfaRun(ctypes.Structure):
    _fields_ = [("start_wv", ctypes.c_double), ("end_wv", ctypes.c_double),
                ("cutoff", ctypes.c_double), ("target", ctypes.c_int),
                ("mol_code", ctypes.c_int), ("chi", ctypes.c_int), ("shape", ctypes.c_int),
                ("precision", ctypes.c_int)]


class MarfaError(RuntimeError):
    """A library call returned a non-zero status; .code is that status (the
    reference's `stop` code where one exists)."""

    def __init__(self, code: int, message: str = ""):
        super().__init__(f"marfa status {code}: {message}")
        self.code = code


_lib = None

P = ctypes.c_void_p
D = ctypes.c_double
I = ctypes.c_int
I64 = ctypes.c_int64


def load():
    """Load the library (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise OSError(f"{LIB_PATH} is missing: build it with `python -m marfa_b200.build`")
    lib = ctypes.CDLL(str(LIB_PATH))
    sig = {
        "marfa_ctx_create": (I, [P, I64, P, I, I, I, ctypes.POINTER(P)]),
        "marfa_ctx_destroy": (None, [P]),
        "marfa_last_error": (ctypes.c_char_p, [P]),
        "marfa_num_subintervals": (I, [D, D]),
        "marfa_record_number": (I, [D, I]),
        "marfa_compute": (I, [P, ctypes.POINTER(MarfaRun), P, P, P, I, P, P]),
        "marfa_compute_batched": (I, [P, ctypes.POINTER(MarfaRun), I, P, P, P, P, P, P]),
        "marfa_compute_device": (I, [P, ctypes.POINTER(MarfaRun), I, P, P, P, P, P, P]),
        "marfa_synchronize": (I, [P]),
        "marfa_eval_count": (I, [P, ctypes.POINTER(MarfaRun), I, P, P, P, P, P]),
        "marfa_debug_accumulators": (I, [P, ctypes.POINTER(MarfaRun), P, P, P, I, I, I, P]),
        "marfa_last_timings": (I, [P, P]),
        "marfa_plan_windows": (I, [P, I64, D, D, D, P, P]),
        "marfa_compute_record_static": (I, [P, I64, P, I, I, ctypes.POINTER(MarfaRun), D, D, D, I, P,
                                            P, ctypes.c_char_p, ctypes.c_size_t]),
        "marfa_ctx_set_line_params": (I, [P, P, P]),
        "marfa_ctx_set_tips_grid": (I, [P, D, D]),
        "marfa_vjp": (I, [P, ctypes.POINTER(MarfaRun), P, P, P, I, P, P, P, P, P]),
        "marfa_graph_create": (I, [P, ctypes.POINTER(MarfaRun), I, P, P, P, P, P, ctypes.POINTER(P)]),
        "marfa_graph_launch": (I, [P, P, P, P, P]),
        "marfa_graph_destroy": (None, [P]),
        "marfa_autotune": (I, [P, ctypes.POINTER(MarfaRun), I, P, P, P, P, P]),
        "marfa_ctx_set_launch": (I, [P, I, I, I]),
        "marfa_ctx_get_launch": (I, [P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
