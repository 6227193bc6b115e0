"""ctypes wrapper of the CPU oracle (oracle/cortado_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke() entry point as a
checker, and by bench.py's CPU-baseline legs.  The product library never uses
it.  All functions take and return numpy arrays / bytes.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcortado_oracle.so")
CS = 16384

STATUS = {0: "OK", 1: "EB_TOO_SMALL", 2: "EB_TOO_LARGE", 3: "CORRUPT_STREAM",
          4: "SIZE_MISMATCH", 7: "INVALID_ARG", 10: "CAPACITY"}


class OracleError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"oracle {what}: {STATUS.get(code, code)}")
        self.code = code


def build() -> str:
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "cortado_oracle.c")):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(build())
        u8p = ctypes.POINTER(ctypes.c_uint8)
        i64 = ctypes.c_int64
        i64p = ctypes.POINTER(ctypes.c_int64)
        f32 = ctypes.c_float
        c_int = ctypes.c_int
        fp = ctypes.POINTER(ctypes.c_float)
        L.ora_store_encode.argtypes = [u8p, i64, f32, u8p, i64, i64p, c_int]
        L.ora_store_decode.argtypes = [u8p, i64, u8p, i64, i64p, c_int]
        L.ora_init_recv.argtypes = [u8p, i64, u8p, i64, i64p, c_int]
        L.ora_init_send.argtypes = [u8p, i64, f32, u8p, i64, i64p, c_int]
        L.ora_resi_send.argtypes = [u8p, i64, f32, f32, u8p, i64, i64p, c_int]
        L.ora_resi_recv.argtypes = [u8p, i64, u8p, i64, u8p, i64, i64p, c_int]
        L.ora_client_roundtrip.argtypes = [fp, i64, f32, fp]
        L.ora_maxabs.argtypes = [fp, fp, i64, f32]
        L.ora_maxabs.restype = i64
        L.ora_max_stream_bytes.argtypes = [i64]
        L.ora_max_stream_bytes.restype = i64
        L.ora_eb_params.argtypes = [f32, ctypes.POINTER(c_int), ctypes.POINTER(c_int), ctypes.POINTER(c_int)]
        L.ora_bit4.argtypes = [u8p, u8p, c_int]
        L.ora_ibit4.argtypes = [u8p, u8p, c_int]
        L.ora_rze.argtypes = [u8p, c_int, u8p]
        L.ora_irze.argtypes = [u8p, c_int, u8p]
        for n in ("ora_sq", "ora_cq", "ora_iq"):
            getattr(L, n).argtypes = [ctypes.c_uint32, c_int]
            getattr(L, n).restype = ctypes.c_uint32
        _lib = L
    return _lib


def _u8(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def _bytes(x) -> np.ndarray:
    if isinstance(x, (bytes, bytearray)):
        return np.frombuffer(bytes(x), dtype=np.uint8)
    return np.ascontiguousarray(x).view(np.uint8).reshape(-1)


def _threads(t):
    return int(t) if t else (os.cpu_count() or 1)


def max_stream_bytes(n_bytes: int) -> int:
    return int(lib().ora_max_stream_bytes(n_bytes))


def eb_params(eb: float):
    e, t, o = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    st = lib().ora_eb_params(ctypes.c_float(eb), ctypes.byref(e), ctypes.byref(t), ctypes.byref(o))
    if st:
        raise OracleError(st, "eb")
    return e.value, t.value, o.value


def store_encode(x, eb_abs: float, threads: int | None = None) -> bytes:
    b = _bytes(x)
    cap = max_stream_bytes(b.size)
    out = np.empty(cap, np.uint8)
    sz = ctypes.c_int64()
    st = lib().ora_store_encode(_u8(b), b.size, eb_abs, _u8(out), cap, ctypes.byref(sz), _threads(threads))
    if st:
        raise OracleError(st, "store_encode")
    return out[: sz.value].tobytes()


def _decode(fn, stream, threads) -> np.ndarray:
    s = _bytes(stream)
    n = int(np.frombuffer(s[:8].tobytes(), np.int64)[0]) if s.size >= 8 else 0
    out = np.empty(max(n, 1), np.uint8)
    sz = ctypes.c_int64()
    st = fn(_u8(s), s.size, _u8(out), max(n, 0), ctypes.byref(sz), _threads(threads))
    if st:
        raise OracleError(st, fn.__name__)
    return out[: sz.value].view(np.float32) if sz.value % 4 == 0 else out[: sz.value]


def store_decode(stream, threads=None) -> np.ndarray:
    return _decode(lib().ora_store_decode, stream, threads)


def init_recv(stream, threads=None) -> np.ndarray:
    return _decode(lib().ora_init_recv, stream, threads)


def init_send(stored, request_eb_abs: float, threads=None) -> bytes:
    s = _bytes(stored)
    n = int(np.frombuffer(s[:8].tobytes(), np.int64)[0])
    cap = max_stream_bytes(n)
    out = np.empty(cap, np.uint8)
    sz = ctypes.c_int64()
    st = lib().ora_init_send(_u8(s), s.size, request_eb_abs, _u8(out), cap, ctypes.byref(sz), _threads(threads))
    if st:
        raise OracleError(st, "init_send")
    return out[: sz.value].tobytes()


def resi_send(stored, src_eb_abs: float, dst_eb_abs: float, threads=None) -> bytes:
    s = _bytes(stored)
    n = int(np.frombuffer(s[:8].tobytes(), np.int64)[0])
    cap = max_stream_bytes(n)
    out = np.empty(cap, np.uint8)
    sz = ctypes.c_int64()
    st = lib().ora_resi_send(_u8(s), s.size, src_eb_abs, dst_eb_abs, _u8(out), cap, ctypes.byref(sz), _threads(threads))
    if st:
        raise OracleError(st, "resi_send")
    return out[: sz.value].tobytes()


def resi_recv(src, resi, threads=None) -> np.ndarray:
    a = _bytes(src)
    r = _bytes(resi)
    out = np.empty(max(a.size, 1), np.uint8)
    sz = ctypes.c_int64()
    st = lib().ora_resi_recv(_u8(a), a.size, _u8(r), r.size, _u8(out), a.size, ctypes.byref(sz), _threads(threads))
    if st:
        raise OracleError(st, "resi_recv")
    return out[: sz.value].view(np.float32)


def client_roundtrip(x, eb_abs: float) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.float32).reshape(-1)
    out = np.empty_like(a)
    fp = ctypes.POINTER(ctypes.c_float)
    st = lib().ora_client_roundtrip(a.ctypes.data_as(fp), a.size, eb_abs, out.ctypes.data_as(fp))
    if st:
        raise OracleError(st, "client_roundtrip")
    return out


def maxabs(recon, orig, eb: float) -> int:
    """-1 when every value is within eb (MAXABS_f32 rules), else the first bad index."""
    r = np.ascontiguousarray(recon, dtype=np.float32).reshape(-1)
    o = np.ascontiguousarray(orig, dtype=np.float32).reshape(-1)
    assert r.size == o.size
    fp = ctypes.POINTER(ctypes.c_float)
    return int(lib().ora_maxabs(r.ctypes.data_as(fp), o.ctypes.data_as(fp), r.size, eb))


def bit4(chunk: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(chunk, dtype=np.uint8)
    out = np.empty(a.size, np.uint8)
    lib().ora_bit4(_u8(a), _u8(out), a.size)
    return out


def ibit4(chunk: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(chunk, dtype=np.uint8)
    out = np.empty(a.size, np.uint8)
    lib().ora_ibit4(_u8(a), _u8(out), a.size)
    return out


def rze(chunk: np.ndarray):
    a = np.zeros(CS + 64, np.uint8)
    a[: chunk.size] = chunk
    out = np.zeros(CS + 64, np.uint8)
    c = lib().ora_rze(_u8(a), int(chunk.size), _u8(out))
    return None if c < 0 else out[:c].copy()


def irze(payload: np.ndarray):
    a = np.zeros(CS + 64, np.uint8)
    a[: payload.size] = payload
    out = np.zeros(CS + 64, np.uint8)
    c = lib().ora_irze(_u8(a), int(payload.size), _u8(out))
    return None if c < 0 else out[:c].copy()


def sq(v: int, eb_e: int) -> int:
    return int(lib().ora_sq(v & 0xFFFFFFFF, eb_e))


def cq(v: int, eb_e: int) -> int:
    return int(lib().ora_cq(v & 0xFFFFFFFF, eb_e))


def iq(v: int, eb_e: int) -> int:
    return int(lib().ora_iq(v & 0xFFFFFFFF, eb_e))


def noa_range(x) -> float:
    """max - min in float32, NaNs ignored (the reference uses
    thrust::minmax_element, INOA_f32.h:52-61)."""
    a = np.asarray(x, dtype=np.float32).reshape(-1)
    if a.size == 0:
        return np.float32(0)
    return np.float32(np.nanmax(a)) - np.float32(np.nanmin(a))
