"""Host-side logic of the reference's CLI drivers that surrounds the kernels:
error-bound parsing and NOA scaling, the server storage directory
(``<basename>.stor.NN`` + ``.stor.meta``) and the choice of the stored stream
that serves a request.  Pure Python + numpy; no device code.

Reference: src/cortado_store.cu:153-156 (sort + dedupe), :220-227 (NOA
scaling, halving), :299-314 (file names, metadata); src/cortado_init.cu:287-322
and src/cortado_resi.cu:318-348 (metadata read, request scaling, selection);
include/util.h:70-135 (.stor.meta layout).
"""
from __future__ import annotations

import os
import shutil
import struct
from dataclasses import dataclass

import numpy as np

CS = 16384
HEADER_BYTES = 16


def f32(x) -> np.float32:
    """A bound as the reference's argument parser holds it (float)."""
    if isinstance(x, str):
        return np.float32(float(x))
    return np.float32(x)


def noa_scale(eb, value_range) -> np.float32:
    """eb_abs = range * eb in float32 (cortado_store.cu:222-224)."""
    with np.errstate(over="ignore"):
        return np.float32(np.float32(value_range) * np.float32(eb))


def value_range(vmin, vmax) -> np.float32:
    with np.errstate(over="ignore"):
        return np.float32(np.float32(vmax) - np.float32(vmin))


def store_bounds(ebs, abs_mode: bool, vrange) -> tuple[list[np.float32], list[np.float32]]:
    """User bounds sorted descending and deduplicated on the given values,
    then scaled (NOA) -- returns (user values, absolute values)."""
    user = sorted({f32(e) for e in ebs}, reverse=True)
    absolute = [e if abs_mode else noa_scale(e, vrange) for e in user]
    return user, absolute


def select_stored(server_ebs_abs, request_abs) -> int:
    """First stored bound (descending order) not above the request
    (cortado_init.cu:298-304); -1 if the request is too tight."""
    r = f32(request_abs)
    for i, e in enumerate(server_ebs_abs):
        if r >= np.float32(e):
            return i
    return -1


def stor_name(input_path: str, index: int) -> str:
    return f"{os.path.basename(input_path)}.stor.{index:02d}"


@dataclass
class StorMeta:
    name: str             # input path as given to store
    ebs: list             # absolute bounds, descending (float32)
    range: np.float32     # max - min of the original


def pack_meta(m: StorMeta) -> bytes:
    """util.h:70-99: int32 name_len, int32 n, float32 ebs[n], float32 range, name."""
    name = m.name.encode()
    return (struct.pack("<ii", len(name), len(m.ebs)) + np.asarray(m.ebs, np.float32).tobytes()
            + np.float32(m.range).tobytes() + name)


def unpack_meta(b: bytes) -> StorMeta:
    name_len, n = struct.unpack_from("<ii", b, 0)
    ebs = list(np.frombuffer(b, np.float32, n, 8))
    rng = np.frombuffer(b, np.float32, 1, 8 + 4 * n)[0]
    name = b[12 + 4 * n: 12 + 4 * n + name_len].decode()
    return StorMeta(name, ebs, rng)


def write_storage(out_dir: str, input_path: str, streams, ebs_abs, vrange) -> None:
    """Replaces out_dir (the reference deletes it first, cortado_store.cu:170-179)
    and writes one stream per bound plus .stor.meta."""
    shutil.rmtree(out_dir, ignore_errors=True)
    os.makedirs(out_dir, exist_ok=True)
    for i, s in enumerate(streams):
        with open(os.path.join(out_dir, stor_name(input_path, i)), "wb") as f:
            f.write(bytes(s))
    with open(os.path.join(out_dir, ".stor.meta"), "wb") as f:
        f.write(pack_meta(StorMeta(input_path, list(ebs_abs), np.float32(vrange))))


def read_storage_meta(server_dir: str) -> StorMeta:
    with open(os.path.join(server_dir, ".stor.meta"), "rb") as f:
        return unpack_meta(f.read())


def stream_orig_bytes(stream) -> int:
    """Original size recorded in a stream header."""
    return int(np.frombuffer(bytes(stream[:8]), np.int64)[0])


def chunks_of(n_bytes: int) -> int:
    return (n_bytes + CS - 1) // CS


def max_stream_bytes(n_bytes: int) -> int:
    c = chunks_of(n_bytes)
    return HEADER_BYTES + 2 * c + c * CS


@dataclass
class RequestPlan:
    """What one init/residual request resolves to on the server."""
    stored_index: int
    eb1_abs: np.float32   # init: request bound; residual: source bound
    eb2_abs: np.float32   # residual: destination bound (init: unused)


def plan_init(meta: StorMeta, request_eb, abs_mode: bool) -> RequestPlan:
    req = f32(request_eb) if abs_mode else noa_scale(request_eb, meta.range)
    return RequestPlan(select_stored(meta.ebs, req), req, np.float32(0))


def plan_resi(meta: StorMeta, src_eb, dst_eb, abs_mode: bool) -> RequestPlan:
    src = f32(src_eb) if abs_mode else noa_scale(src_eb, meta.range)
    dst = f32(dst_eb) if abs_mode else noa_scale(dst_eb, meta.range)
    return RequestPlan(select_stored(meta.ebs, dst), src, dst)
