"""ctypes binding of the C ABI in include/chaos_lyap.h.

Loads chaos_oneapi_b200/libchaos_lyap.so, built in-tree by
``python -m chaos_oneapi_b200.build``.  There is no fallback: if the library
is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libchaos_lyap.so")

OK, EINVAL, ENOMODEL, EUNSUPPORTED, ECUDA, ENOMEM = range(6)
POINT_OK, POINT_NONFINITE, POINT_STEP_UNDERFLOW, POINT_MAX_STEPS, POINT_ESCAPED = range(5)
METHOD = {"fd": 0, "var": 1, "qr": 2}
INTEG = {"dverk": 0, "dverk65": 1, "dopri5": 2}
PREC = {"compat": 0, "fp64": 1, "fp32": 2}
GS = {"cgs": 0, "mgs": 1}
LAYOUT = {"point": 0, "comp": 1}
SCHED = {"auto": 0, "direct": 1, "persistent": 2, "split": 3, "split_persistent": 4}


class Desc(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("model", ctypes.c_char * 32),
        ("method", ctypes.c_int32),
        ("integrator", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("gs", ctypes.c_int32),
        ("k", ctypes.c_int32),
        ("layout", ctypes.c_int32),
        ("eps", ctypes.c_double),
        ("h", ctypes.c_double),
        ("rtol", ctypes.c_double),
        ("atol", ctypes.c_double),
        ("h_max", ctypes.c_double),
        ("h_min", ctypes.c_double),
        ("t_transient", ctypes.c_double),
        ("t_align", ctypes.c_double),
        ("t_avg", ctypes.c_double),
        ("dt_renorm", ctypes.c_double),
        ("max_steps", ctypes.c_int64),
        ("device", ctypes.c_int32),
        ("schedule", ctypes.c_int32),
        ("block", ctypes.c_int32),
        ("variant", ctypes.c_int32),
        ("escape", ctypes.c_double),
        ("reserved", ctypes.c_int32 * 4),
    ]


class Segment(ctypes.Structure):
    _fields_ = [("handle", ctypes.c_void_p), ("P", ctypes.c_int64), ("params", ctypes.c_void_p),
                ("inits", ctypes.c_void_p), ("spectrum", ctypes.c_void_p),
                ("status", ctypes.c_void_p), ("steps", ctypes.c_void_p),
                ("t_avg_per_point", ctypes.c_void_p)]


class ChaosError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"chaos_lyap error {code}: {msg}")
        self.code = code


_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)

# name -> (restype, argtypes)
SIGNATURES = {
    "chaos_lyap_abi_version": (ctypes.c_int, []),
    "chaos_lyap_last_error": (ctypes.c_char_p, []),
    "chaos_lyap_desc_init": (ctypes.c_int, [ctypes.POINTER(Desc)]),
    "chaos_lyap_model_count": (ctypes.c_int, []),
    "chaos_lyap_model_name": (ctypes.c_int, [ctypes.c_int, ctypes.c_char_p, ctypes.c_int]),
    "chaos_lyap_query_model": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32),
                                              ctypes.POINTER(ctypes.c_int32),
                                              ctypes.POINTER(ctypes.c_int32)]),
    "chaos_lyap_model_text": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p,
                                             ctypes.c_int]),
    "chaos_lyap_create": (ctypes.c_int, [ctypes.POINTER(Desc), ctypes.POINTER(_P)]),
    "chaos_lyap_destroy": (ctypes.c_int, [_P]),
    "chaos_lyap_run": (ctypes.c_int, [_P, ctypes.c_int64, _P, _P, _P, _P, _P, _P, _P]),
    "chaos_lyap_run_host": (ctypes.c_int, [_P, ctypes.c_int64, _P, _P, _P, _P, _P, _P]),
    "chaos_lyap_sync": (ctypes.c_int, [_P]),
    "chaos_lyap_autotune": (ctypes.c_int, [_P, ctypes.c_int64, _P, _P,
                                           ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_int32)]),
    "chaos_lyap_autotune_map": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_int64, _P, _P,
                                               ctypes.POINTER(ctypes.c_int32),
                                               ctypes.POINTER(ctypes.c_int32)]),
    "chaos_lyap_run_batch": (ctypes.c_int, [ctypes.POINTER(Segment), ctypes.c_int, _P]),
    "chaos_lyap_batch_graph_create": (ctypes.c_int, [ctypes.POINTER(Segment), ctypes.c_int,
                                                     ctypes.POINTER(_P)]),
    "chaos_lyap_graph_launch": (ctypes.c_int, [_P, _P]),
    "chaos_lyap_graph_destroy": (ctypes.c_int, [_P]),
    "chaos_lyap_get_variant": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int32)]),
    "chaos_lyap_trajectory": (ctypes.c_int, [_P, ctypes.c_int64, _P, _P, ctypes.c_int32, _P, _P,
                                             _P, _P, _P]),
    "chaos_lyap_cudaLyapunov": (ctypes.c_int, [
        ctypes.c_int, ctypes.c_int, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        _P, _P, ctypes.c_int32, ctypes.c_char_p, _P, ctypes.c_int32, ctypes.c_double,
        ctypes.c_double, _P, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
        ctypes.c_double, _P]),
    "chaos_lyap_fma_peak": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           ctypes.POINTER(ctypes.c_double)]),
    "chaos_lyap_make_grid": (ctypes.c_int64, [ctypes.c_int32, _D, _D, _D, _D]),
    "chaos_lyap_make_inits": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int64, _D, ctypes.c_double,
                                             ctypes.c_int32, ctypes.c_uint64, _D]),
}


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m chaos_oneapi_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load()


def check(rc: int) -> None:
    if rc != OK:
        raise ChaosError(rc, lib.chaos_lyap_last_error().decode())
