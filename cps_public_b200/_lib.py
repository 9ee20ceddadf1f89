"""ctypes binding of libcpsb200.so (the C ABI declared in include/cpsb200.h).

The library is loaded from the package directory; a missing or unloadable
library raises ImportError -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libcpsb200.so")

CPSB_OK = 0
CPSB_NOT_CONVERGED = 1
WILSON, DWF, MOBIUS, ZMOBIUS = 0, 1, 2, 3
F64, F32, F16 = 0, 1, 2
ORDER_CANONICAL, ORDER_WILSON = 0, 1
MULTI, SINGLE = 0, 1
FERMION_CB, FERMION_4D_EE = 0, 1

SYMBOLS = [
    "cpsb_init", "cpsb_serve_submit_minvcg", "cpsb_error_string", "cpsb_last_error", "cpsb_mem_info", "cpsb_gauge_load", "cpsb_gauge_free", "cpsb_dslash",
    "cpsb_matpc", "cpsb_mdagm", "cpsb_invcg", "cpsb_invcg_multi", "cpsb_minvcg", "cpsb_matinv", "cpsb_fmatinv", "cpsb_dminus", "cpsb_invcg_dev",
    "cpsb_invcg_multi_dev", "cpsb_mdagm_dev", "cpsb_minvcg_dev", "cpsb_dslash_ex", "cpsb_mdagm_ex", "cpsb_bench_dslash",
    "cpsb_kernel_launches", "cpsb_dslash_multi_dev", "cpsb_mdagm_multi_dev",
    "cpsb_redot_noalloc", "cpsb_serve_create", "cpsb_serve_submit", "cpsb_serve_poll", "cpsb_serve_wait",
    "cpsb_serve_stats", "cpsb_serve_destroy", "cpsb_fermion_convert", "cpsb_minresext", "cpsb_minvcg_multi",
    "cpsb_minvcg_multi_dev",
]


class DiracParams(C.Structure):
    _fields_ = [("action", C.c_int), ("ls", C.c_int), ("mass", C.c_double), ("m5", C.c_double),
                ("a5_inv", C.c_double), ("mobius_b", C.c_double), ("mobius_c", C.c_double),
                ("pc_type", C.c_int), ("zmobius_b", C.POINTER(C.c_double)), ("zmobius_c", C.POINTER(C.c_double))]


class CgArg(C.Structure):
    _fields_ = [("stop_rsd", C.c_double), ("max_num_iter", C.c_int), ("precision", C.c_int),
                ("reliable_delta", C.c_double), ("batch", C.c_int)]


class SolveResult(C.Structure):
    _fields_ = [("iters", C.c_int), ("true_rsd", C.c_double), ("iter_rsd", C.c_double),
                ("reliable_updates", C.c_int), ("seconds", C.c_double), ("status", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServeStats(C.Structure):
    _fields_ = [("completed", C.c_long), ("failed", C.c_long), ("rhs_completed", C.c_long),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("max_ms", C.c_double),
                ("requests_per_s", C.c_double), ("rhs_per_s", C.c_double), ("peak_running", C.c_int),
                ("queued", C.c_int), ("running", C.c_int), ("budget_bytes", C.c_double),
                ("peak_reserved_bytes", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_dp = C.POINTER(C.c_double)
_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise ImportError(f"{LIBPATH} is missing: build it with `python -m cps_public_b200.build`")
    lib = C.CDLL(LIBPATH)
    lib.cpsb_error_string.restype = C.c_char_p
    lib.cpsb_last_error.restype = C.c_char_p
    lib.cpsb_init.argtypes = [C.c_int]
    lib.cpsb_mem_info.argtypes = [C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]
    lib.cpsb_gauge_load.argtypes = [C.POINTER(C.c_void_p), _dp, C.POINTER(C.c_int), C.c_int, C.c_int]
    lib.cpsb_gauge_free.argtypes = [C.c_void_p]
    P = C.POINTER(DiracParams)
    A = C.POINTER(CgArg)
    R = C.POINTER(SolveResult)
    lib.cpsb_dslash.argtypes = [C.c_void_p, P, _dp, _dp, C.c_int, C.c_int]
    lib.cpsb_matpc.argtypes = [C.c_void_p, P, _dp, _dp, C.c_int]
    lib.cpsb_mdagm.argtypes = [C.c_void_p, P, _dp, _dp, _dp]
    lib.cpsb_invcg.argtypes = [C.c_void_p, P, A, _dp, _dp, R]
    lib.cpsb_invcg_multi.argtypes = [C.c_void_p, P, A, C.c_int, C.POINTER(_dp), C.POINTER(_dp), R]
    lib.cpsb_minvcg.argtypes = [C.c_void_p, P, A, C.POINTER(_dp), _dp, _dp, C.c_int, _dp, C.c_int, _dp, R]
    lib.cpsb_matinv.argtypes = [C.c_void_p, P, A, _dp, _dp, R]
    lib.cpsb_fmatinv.argtypes = [C.c_void_p, P, A, _dp, _dp, C.c_int, R]
    lib.cpsb_dminus.argtypes = [C.c_void_p, P, _dp, _dp]
    lib.cpsb_invcg_dev.argtypes = [C.c_void_p, P, A, C.c_void_p, C.c_void_p, R, C.c_void_p]
    lib.cpsb_invcg_multi_dev.argtypes = [C.c_void_p, P, A, C.c_int, C.c_void_p, C.c_void_p, R, C.c_void_p]
    lib.cpsb_mdagm_dev.argtypes = [C.c_void_p, P, C.c_void_p, C.c_void_p, _dp, C.c_void_p]
    lib.cpsb_minvcg_dev.argtypes = [C.c_void_p, P, A, C.POINTER(C.c_void_p), C.c_void_p, _dp, C.c_int, _dp, C.c_int,
                                    _dp, R, C.c_void_p]
    lib.cpsb_minvcg_multi.argtypes = [C.c_void_p, P, A, C.c_int, C.POINTER(_dp), C.POINTER(_dp), _dp, C.c_int, _dp,
                                      C.c_int, _dp, R]
    lib.cpsb_minvcg_multi_dev.argtypes = [C.c_void_p, P, A, C.c_int, C.POINTER(C.c_void_p), C.c_void_p, _dp, C.c_int,
                                          _dp, C.c_int, _dp, R, C.c_void_p]
    lib.cpsb_dslash_ex.argtypes = [C.c_void_p, P, C.c_int, _dp, _dp, C.c_int, C.c_int]
    lib.cpsb_mdagm_ex.argtypes = [C.c_void_p, P, C.c_int, _dp, _dp, _dp]
    lib.cpsb_dslash_multi_dev.argtypes = [C.c_void_p, P, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                          C.c_void_p]
    lib.cpsb_mdagm_multi_dev.argtypes = [C.c_void_p, P, C.c_int, C.c_int, C.c_void_p, C.c_void_p, _dp, C.c_void_p]
    lib.cpsb_serve_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_double, C.c_ulonglong]
    lib.cpsb_serve_submit.argtypes = [C.c_void_p, C.c_void_p, P, A, C.c_int, C.POINTER(_dp), C.POINTER(_dp),
                                      C.POINTER(C.c_ulonglong)]
    lib.cpsb_serve_submit_minvcg.argtypes = [C.c_void_p, C.c_void_p, P, A, C.POINTER(_dp), _dp, _dp, C.c_int, _dp,
                                             C.c_int, _dp, C.POINTER(C.c_ulonglong)]
    lib.cpsb_serve_poll.argtypes = [C.c_void_p, C.c_ulonglong, C.POINTER(C.c_int)]
    lib.cpsb_serve_wait.argtypes = [C.c_void_p, C.c_ulonglong, R, _dp]
    lib.cpsb_serve_stats.argtypes = [C.c_void_p, C.POINTER(ServeStats)]
    lib.cpsb_serve_destroy.argtypes = [C.c_void_p]
    lib.cpsb_fermion_convert.argtypes = [C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                         C.c_void_p]
    lib.cpsb_minresext.argtypes = [C.c_void_p, P, _dp, _dp, C.POINTER(_dp), C.POINTER(_dp), C.c_int, _dp]
    lib.cpsb_redot_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_void_p, C.c_void_p]
    lib.cpsb_kernel_launches.argtypes = [C.POINTER(C.c_ulonglong)]
    lib.cpsb_bench_dslash.argtypes = [C.c_void_p, P, C.c_int, C.c_int, C.c_int, _dp, _dp]
    _lib = lib
    return lib


class CpsbError(RuntimeError):
    def __init__(self, code, where):
        lib = load()
        msg = lib.cpsb_error_string(code).decode()
        detail = lib.cpsb_last_error().decode()
        super().__init__(f"{where}: {msg} ({code}) {detail}")
        self.code = code


def check(code, where):
    if code < 0:
        raise CpsbError(code, where)
    return code


def ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)
