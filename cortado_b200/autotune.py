"""Autotuner for the processing parameters of the encode/decode kernels.

Only parameters that change speed, never output bytes, are tuned:

* CTAs per SM of each operation's persistent grid (``cortado_set_launch_ctas``;
  the batched launches of an operation use the same setting): latency hiding
  against shared-memory and L2 pressure;
* for the three encoders, whether the helper CTA's resolver warp turns
  published chunk sizes into inclusive prefixes ahead of the flushes
  (``cortado_set_resolver``), or each flush walks the lookback words itself.

Not tuned, because they are fixed by the format or the register layout: the
chunk size (16 KiB, part of every stream), threads per chunk (128: one
32-word group per thread), and the lookback window (32 words, one per lane;
wider windows measured slower and need a different register layout).

``tune(codec, n_bytes)`` sweeps the parameters per operation on the
benchmark's kind of field (seeded sinusoid with 0.1% outliers, NOA flow) of
the given size and keeps the fastest; results are keyed by GPU name and size
class.  ``apply(codec, n_bytes)`` sets the chosen parameters on a context:
from the user cache (``CORTADO_TUNE_CACHE`` or ~/.cache/cortado_b200), else
from the table shipped for the GPU (``cortado_b200/tuning/*.json``), else the
built-in defaults; it tunes only when asked (``tune_on_miss``).  Codec
creation applies the table for the default size class.
"""
from __future__ import annotations

import json
import os
import statistics

import torch

from . import fields, storage
from .ops import Codec, max_stream_bytes

OPS = ("store", "init_send", "init_recv", "resi_send", "resi_recv")
ENCODERS = ("store", "init_send", "resi_send")
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_CLASS = "le512MiB"
TIE = 0.03  # relative spread of sweep times treated as equal (repeat sweeps differ by 1-2%)


def cache_path() -> str:
    return os.environ.get("CORTADO_TUNE_CACHE") or os.path.join(
        os.environ.get("XDG_CACHE_HOME", os.path.expanduser("~/.cache")), "cortado_b200", "tune.json")


def size_class(n_bytes: int) -> str:
    mb = n_bytes / 2**20
    for lim, name in ((4, "le4MiB"), (64, "le64MiB"), (512, "le512MiB")):
        if mb <= lim:
            return name
    return "gt512MiB"


def gpu_name(device) -> str:
    return torch.cuda.get_device_name(device)


def key(device, n_bytes: int) -> str:
    return f"{gpu_name(device)}|{size_class(n_bytes)}"


def shipped_path(device) -> str:
    name = "".join(ch if ch.isalnum() else "_" for ch in gpu_name(device))
    return os.path.join(HERE, "tuning", name + ".json")


def _time(fn, reps):
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        ts.append(s.elapsed_time(e))
    return statistics.median(ts)


def set_params(codec: Codec, params: dict) -> None:
    """Applies {op: {"ctas_per_sm": n, "resolver": 0/1}} to a context."""
    for op, v in params.items():
        codec.set_launch_ctas(op, int(v.get("ctas_per_sm", 0)))
        if op in ENCODERS and "resolver" in v:
            codec.set_resolver(op, bool(v["resolver"]))


def choose(results: dict) -> tuple:
    """The setting kept from a sweep {(ctas_per_sm, resolver): ms}: settings
    within TIE of the fastest count as equal (the sweep's own noise), and
    among them the most CTAs per SM wins, then the resolver on, since small
    fields and batched launches gain from occupancy more than the tuning
    field shows."""
    fastest = min(results.values())
    return max(k for k, v in results.items() if v <= fastest * (1 + TIE))


def tune(codec: Codec, n_bytes: int = 128 << 20, ctas=(3, 4, 5, 6), reps: int = 5) -> dict:
    """Sweeps every operation's parameters on a seeded sinusoid + 0.1%
    outliers field of n_bytes at NOA 1e-4 (store), 1e-2 (init) and
    1e-2 -> 1e-4 (residual); returns {op: {"ctas_per_sm", "resolver", "ms",
    "sweep_ms"}} and leaves the best setting applied."""
    dev = codec.device
    side = max(1, n_bytes // (4 * 512 * 512))
    x = fields.sinusoid((side, 512, 512), 2, outlier_frac=1e-3, device=dev).reshape(-1)
    n = x.numel() * 4
    lo, hi = codec.INOA_find_range(x)
    rng = storage.value_range(lo, hi)
    eb_s, eb_i, eb_d = (float(storage.noa_scale(e, rng)) for e in ("1e-4", "1e-2", "1e-4"))
    cap = max_stream_bytes(n)
    stor, init, resi = (torch.empty(cap, dtype=torch.uint8, device=dev) for _ in range(3))
    cl, fin = torch.empty_like(x), torch.empty_like(x)
    sz = torch.zeros(8, dtype=torch.int64, device=dev)
    calls = {
        "store": lambda: codec.server_encode(x, n, stor, sz[0:1], eb_s),
        "init_send": lambda: codec.s2c_encode(stor, init, sz[1:2], eb_i, n),
        "init_recv": lambda: codec.client_decode(init, cl, sz[2:3]),
        "resi_send": lambda: codec.residual_encode(stor, resi, sz[3:4], eb_i, eb_d, n),
        "resi_recv": lambda: codec.residual_apply(cl, n, resi, fin, sz[4:5]),
    }
    for op in OPS:  # valid inputs for every later op
        calls[op]()
    codec.sync()
    best = {}
    for op in OPS:
        results = {}
        for resolver in ((1, 0) if op in ENCODERS else (1,)):
            if op in ENCODERS:
                codec.set_resolver(op, bool(resolver))
            for c in ctas:
                codec.set_launch_ctas(op, c)
                results[(c, resolver)] = _time(calls[op], reps)
        c, resolver = choose(results)
        ms = results[(c, resolver)]
        best[op] = {"ctas_per_sm": int(c), "resolver": int(resolver), "ms": ms,
                    "sweep_ms": {f"{k[0]}/{k[1]}": v for k, v in sorted(results.items())}}
        set_params(codec, {op: best[op]})
    codec.sync()
    return best


def _load(path) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def load_cache() -> dict:
    return _load(cache_path())


def save_cache(d: dict) -> None:
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def lookup(device, n_bytes: int):
    """(params, source) for a device and input size: the user cache, then the
    table shipped for this GPU, else (None, "defaults")."""
    k = key(device, n_bytes)
    c = load_cache()
    if k in c:
        return c[k], "cache"
    shipped = _load(shipped_path(device))
    sc = size_class(n_bytes)
    if sc in shipped:
        return shipped[sc], "shipped"
    return None, "defaults"


def apply(codec: Codec, n_bytes: int | None = None, tune_on_miss: bool = False) -> dict:
    """Sets the tuned parameters for inputs of n_bytes (default size class
    when None) on the context and returns {"params", "source"}."""
    nb = n_bytes if n_bytes is not None else 256 << 20
    params, source = lookup(codec.device, nb)
    if params is None and tune_on_miss:
        params = tune(codec, n_bytes=min(max(nb, 1 << 20), 512 << 20))
        c = load_cache()
        c[key(codec.device, nb)] = params
        save_cache(c)
        source = "tuned"
    if params is not None:
        set_params(codec, params)
    return {"params": params, "source": source}
