"""ctypes binding of libcortado.so (the C ABI declared in include/cortado.h).

The library is built in-tree by __graft_entry__.build() / cortado_b200.build.
There is no fallback: if the library is missing, importing this module fails.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# CORTADO_LIB selects another build of the same library (e.g. a tuning variant).
LIB_PATH = os.environ.get("CORTADO_LIB") or os.path.join(HERE, "libcortado.so")

STATUS_NAMES = {
    0: "OK", 1: "EB_TOO_SMALL", 2: "EB_TOO_LARGE", 3: "CORRUPT_STREAM", 4: "SIZE_MISMATCH",
    5: "TIMEOUT", 6: "OOM", 7: "INVALID_ARG", 8: "CUDA", 9: "ALIGNMENT", 10: "CAPACITY", 11: "SCRATCH_LIMIT",
}

# Every symbol include/cortado.h declares, with (restype, argtypes).
_vp, _i64, _f32, _int = ctypes.c_void_p, ctypes.c_int64, ctypes.c_float, ctypes.c_int
SIGNATURES = {
    "cortado_status_string": (ctypes.c_char_p, [_int]),
    "cortado_max_stream_bytes": (_i64, [_i64]),
    "cortado_eb_exponent": (_int, [_f32, ctypes.POINTER(_int)]),
    "cortado_create": (_int, [ctypes.POINTER(_vp), _int]),
    "cortado_destroy": (None, [_vp]),
    "cortado_set_timeout": (_int, [_vp, ctypes.c_uint64]),
    "cortado_sync": (_int, [_vp, _vp]),
    "cortado_store_encode": (_int, [_vp, _vp, _i64, _f32, _vp, _i64, _vp, _vp]),
    "cortado_store_decode": (_int, [_vp, _vp, _i64, _vp, _i64, _vp, _vp]),
    "cortado_init_send": (_int, [_vp, _vp, _i64, _i64, _f32, _vp, _i64, _vp, _vp]),
    "cortado_init_recv": (_int, [_vp, _vp, _i64, _vp, _i64, _vp, _vp]),
    "cortado_resi_send": (_int, [_vp, _vp, _i64, _i64, _f32, _f32, _vp, _i64, _vp, _vp]),
    "cortado_resi_recv": (_int, [_vp, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _vp]),
    "cortado_noa_range": (_int, [_vp, _vp, _i64, ctypes.POINTER(_f32), ctypes.POINTER(_f32), _vp]),
    "cortado_store_encode_noalloc": (_int, [_vp, _i64, _f32, _vp, _i64, _vp, _vp]),
    "cortado_batch": (_int, [_vp, _int, _vp, _int, _vp]),
    "cortado_verify_bound": (_int, [_vp, _vp, _vp, _i64, _f32, _vp, _vp]),
    "cortado_set_launch_ctas": (_int, [_vp, _int, _int]),
    "cortado_set_resolver": (_int, [_vp, _int, _int]),
    "cortado_reserve": (_int, [_vp, _i64, _int]),
    "cortado_selftest_timeout": (_int, [_vp, _vp]),
    "cortado_init_send_apply": (_int, [_vp, _vp, _i64, _i64, _f32, _vp, _i64, _vp, _vp, _vp]),
    "cortado_noa_range_device": (_int, [_vp, _vp, _i64, _vp, _vp]),
    "cortado_store_encode_noa": (_int, [_vp, _vp, _i64, _vp, _f32, _vp, _i64, _vp, _vp]),
    "cortado_init_send_noa": (_int, [_vp, _vp, _i64, _i64, _vp, _f32, _vp, _i64, _vp, _vp]),
    "cortado_resi_send_noa": (_int, [_vp, _vp, _i64, _i64, _vp, _f32, _f32, _vp, _i64, _vp, _vp]),
    "cortado_resi_send_apply": (_int, [_vp, _vp, _i64, _i64, _f32, _f32, _vp, _i64, _vp, _vp, _vp]),
    "cortado_init_send_apply_noa": (_int, [_vp, _vp, _i64, _i64, _vp, _f32, _vp, _i64, _vp, _vp, _vp]),
    "cortado_resi_send_apply_noa": (_int, [_vp, _vp, _i64, _i64, _vp, _f32, _f32, _vp, _i64, _vp, _vp, _vp]),
}

OPS = {"store": 0, "init_send": 1, "resi_send": 2, "store_decode": 3, "init_recv": 4, "resi_recv": 5,
       "init_send_apply": 6, "resi_send_apply": 7}


class Item(ctypes.Structure):
    """cortado_item (include/cortado.h)."""
    _fields_ = [("d_in", ctypes.c_void_p), ("in_bytes", ctypes.c_int64), ("n_bytes", ctypes.c_int64),
                ("eb1", ctypes.c_float), ("eb2", ctypes.c_float), ("d_src", ctypes.c_void_p),
                ("d_out", ctypes.c_void_p), ("out_capacity", ctypes.c_int64), ("d_outsize", ctypes.c_void_p)]


class CortadoError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = int(code)
        self.name = STATUS_NAMES.get(self.code, str(code))
        super().__init__(f"{what}: {self.name}" if what else self.name)


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libcortado.so not built ({LIB_PATH}); run __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, what: str = "") -> None:
    if status:
        raise CortadoError(status, what)
