"""ctypes binding of libamls_b200.so (the C ABI declared in include/amls_b200.h).

Loading fails loudly: there is no pure-Python or CPU fallback for any entry
point of the library.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libamls_b200.so")

AMLS_OK = 0
AMLS_ERR_INVALID_ARGUMENT = 1
AMLS_ERR_NOT_SPD = 2
AMLS_ERR_ITERATION = 3
AMLS_ERR_TIMEOUT = 4
AMLS_ERR_OOM = 5
AMLS_ERR_CUDA = 6
AMLS_ERR_NUMERIC = 7
AMLS_ERR_PARTITION = 8
AMLS_ERR_NO_DEVICE = 9

T_SLOTS = 8
INFO_SLOTS = 16
WORK_SLOTS = 8
TIMING_KEYS = ["partition", "upload", "elimination", "condense", "reduced", "backtransform", "total",
               "device"]
PROF_CATS = ["cholesky", "trsm", "gemm", "front_update", "tridiag", "bisect", "inverse_iter",
             "eigvec_backtransform", "other"]

# every function the header declares (checked by the CPU tests)
EXPORTS = [
    "amls_options_default", "amls_create", "amls_destroy", "amls_last_error", "amls_partition",
    "amls_solve", "amls_analyze", "amls_solve_values", "amls_info", "amls_work",
    "amls_sygvx_batched", "amls_set_profiling", "amls_kernel_times", "amls_category_work",
    "amls_sygvx_lowest_noalloc", "amls_sensitivities", "amls_permutation", "amls_solve_batch",
    "amls_analyze_batch", "amls_solve_values_batch", "amls_mm_read", "amls_mm_write",
    "amls_eliminate", "amls_condense", "amls_pass_modes", "amls_reduced_eig", "amls_backtransform",
    "amls_refine", "amls_tree", "amls_element_pattern", "amls_hex_assemble",
]
NOALLOC_MAX_N = 128


class Options(C.Structure):
    """amls_options (field order and types of the C struct)."""
    _fields_ = [
        ("nLevels", C.c_int32), ("twoPass", C.c_int32), ("leafSize", C.c_int64),
        ("thresholdFactor", C.c_double), ("fixedKeep", C.c_int64), ("nev", C.c_int64),
        ("denseProjectedMax", C.c_int64), ("shift", C.c_double), ("numThreads", C.c_int32),
        ("recoverVectors", C.c_int32), ("verbosity", C.c_int32), ("refine", C.c_int32),
        ("refineMaxIter", C.c_int32), ("refineExtra", C.c_int32), ("refineTol", C.c_double),
        ("precision", C.c_int32), ("silMode", C.c_int32),
    ]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libamls_b200.so not built ({LIB_PATH}); run amls_b200.build.build()")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        L.amls_last_error.restype = C.c_char_p
        L.amls_options_default.argtypes = [C.POINTER(Options)]
        L.amls_create.argtypes = [C.c_int, C.POINTER(P)]
        L.amls_destroy.argtypes = [P]
        L.amls_partition.argtypes = [C.c_int64, i64p, i32p, i64p, i32p, C.c_int32, C.c_int64,
                                     i64p, C.POINTER(C.c_int64), i64p, i32p, i64p, i64p, i64p, i64p]
        L.amls_solve.argtypes = [P, C.c_int64, P, P, P, P, P, P, C.POINTER(Options), P, P,
                                 C.POINTER(C.c_int64), P]
        L.amls_analyze.argtypes = [P, C.c_int64, P, P, P, P, C.POINTER(Options)]
        L.amls_solve_values.argtypes = [P, P, P, C.c_int32, P, P, C.c_int32,
                                        C.POINTER(C.c_int64), P]
        L.amls_info.argtypes = [P, P]
        L.amls_set_profiling.argtypes = [P, C.c_int32]
        L.amls_kernel_times.argtypes = [P, P, P]
        L.amls_category_work.argtypes = [P, P, P]
        L.amls_sensitivities.argtypes = [P, C.c_int64, C.c_int32, P, C.c_int32, P, P, P, P,
                                         C.c_double, P, P, P, P, P]
        L.amls_sygvx_lowest_noalloc.argtypes = [C.c_int64, P, P, C.c_int64, P, P,
                                                C.POINTER(C.c_int64), P]
        L.amls_work.argtypes = [P, P]
        L.amls_permutation.argtypes = [P, P]
        L.amls_eliminate.argtypes = [P, P, P, C.c_int32]
        L.amls_condense.argtypes = [P, C.c_int32, C.c_int64, C.c_double, C.POINTER(C.c_int64)]
        L.amls_pass_modes.argtypes = [P, P, P]
        L.amls_reduced_eig.argtypes = [P, C.c_int64, C.c_int32, P, C.POINTER(C.c_int64)]
        L.amls_backtransform.argtypes = [P, P, C.c_int32, C.POINTER(C.c_int64)]
        L.amls_refine.argtypes = [P, C.c_int64, P, P, C.c_int32, C.POINTER(C.c_int64)]
        L.amls_tree.argtypes = [P, C.POINTER(C.c_int64), P, P, P]
        L.amls_element_pattern.argtypes = [C.c_int64, C.c_int64, C.c_int32, P, C.POINTER(C.c_int64), P, P]
        L.amls_hex_assemble.argtypes = [P, C.c_int32, C.c_int64, C.c_int64, P, P, P, P, P, C.c_double, C.c_int64,
                                        P, P, P, P, C.c_int32]
        L.amls_mm_read.argtypes = [C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), P, P, P]
        L.amls_mm_write.argtypes = [C.c_char_p, C.c_int64, P, P, P]
        L.amls_solve_batch.argtypes = [P, C.c_int32, P, P, P, P, P, P, P, C.POINTER(Options), P, P, P, P]
        L.amls_analyze_batch.argtypes = [P, C.c_int32, P, P, P, P, P, C.POINTER(Options)]
        L.amls_solve_values_batch.argtypes = [P, P, P, C.c_int32, P, P, P, C.c_int32, P]
        L.amls_sygvx_batched.argtypes = [P, C.c_int32, P, P, P, P, C.c_int32, C.c_int64,
                                         C.c_int64, C.c_double, C.c_double, P, P, P, P, P, P]
        _lib = L
    return _lib


class AmlsStatusError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[amls status {code}] {msg}")
        self.code = code


class NotSPDError(AmlsStatusError):
    pass


def check(code: int) -> None:
    if code == AMLS_OK:
        return
    msg = lib().amls_last_error().decode(errors="replace")
    if code == AMLS_ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if code == AMLS_ERR_NOT_SPD:
        raise NotSPDError(code, msg)
    raise AmlsStatusError(code, msg)


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)
