"""Host mirror of the reference's operator interface for the encode/decode path.

The reference exposes header-only host wrappers that take device buffers
(include/d_server_encode.h:146 ``d_server_encode``, :263 ``d_server_decode``,
include/d_s2c.h:203 ``d_s2c_encode``, include/d_client_encode.h:262
``d_client_decode``, include/d_residual_encode.h:204 ``d_residual_encode``,
:350 ``d_residual_apply``, include/preprocessors/include/INOA_f32.h:52
``d_INOA_find_range``).  ``Codec`` offers the same operations with the same
argument meaning on torch CUDA tensors, calling libcortado's C ABI:

* bounds are absolute float32 values (the callers do the NOA scaling, as the
  reference's CLIs do); ``server_encode`` halves its bound for the stored bins;
* output sizes are written to a device int64 (``d_outsize``), as in the
  reference;
* error-bound problems raise ``CortadoError`` (the reference throws
  ``std::runtime_error("LC error")``); problems the device detects are raised by
  ``sync()`` (the reference traps).

The ``store``/``init_send``/... convenience methods allocate their outputs,
synchronize and return trimmed tensors.
"""
from __future__ import annotations

import ctypes

import torch

from . import _native
from ._native import CortadoError, check

CS = 16384


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _nbytes(t: torch.Tensor) -> int:
    return t.numel() * t.element_size()


def _stream(stream) -> int | None:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, torch.cuda.Stream):
        return stream.cuda_stream
    return int(stream)


def max_stream_bytes(n_bytes: int) -> int:
    return int(_native.lib().cortado_max_stream_bytes(n_bytes))


def eb_exponent(eb_abs: float) -> int:
    e = ctypes.c_int()
    check(_native.lib().cortado_eb_exponent(float(eb_abs), ctypes.byref(e)), "error bound")
    return e.value


class Codec:
    """One libcortado context (scratch for one stream at a time) on a device."""

    def __init__(self, device: int | torch.device | None = None, tuned: bool = True):
        """tuned: set the autotuner's launch parameters for this GPU (the user
        cache, else the table shipped for it; see cortado_b200.autotune)."""
        if not torch.cuda.is_available():
            raise RuntimeError("cortado_b200 needs a CUDA device")
        if device is None:
            device = torch.cuda.current_device()
        self.device = torch.device("cuda", device if isinstance(device, int) else device.index or 0)
        self._L = _native.lib()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(self._L.cortado_create(ctypes.byref(h), self.device.index), "cortado_create")
        self._h = h
        self.tuning = {"params": None, "source": "defaults"}
        if tuned:
            from . import autotune
            self.tuning = autotune.apply(self)

    def close(self):
        if getattr(self, "_h", None):
            self._L.cortado_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_timeout(self, seconds: float):
        check(self._L.cortado_set_timeout(self._h, int(seconds * 1e9)), "set_timeout")

    def selftest_timeout(self, stream=None):
        """Enqueues a bounded device wait that cannot succeed; the next sync()
        raises CortadoError TIMEOUT once the context's timeout has passed."""
        check(self._L.cortado_selftest_timeout(self._h, _stream(stream)), "selftest_timeout")

    def reserve(self, chunks: int, items: int = 0):
        """Sizes the scratch for calls of up to `chunks` chunks (all items of a
        batched call together) and `items` batch items, so that no later call
        allocates device memory."""
        check(self._L.cortado_reserve(self._h, int(chunks), int(items)), "reserve")

    def set_launch_ctas(self, op: str, ctas_per_sm: int):
        """Persistent-grid size of one operation (0 = occupancy limit)."""
        check(self._L.cortado_set_launch_ctas(self._h, _native.OPS[op], int(ctas_per_sm)), "set_launch_ctas")

    def set_resolver(self, op: str, enabled: bool):
        """Lookback resolver warp of an encoder's launches on or off."""
        check(self._L.cortado_set_resolver(self._h, _native.OPS[op], int(bool(enabled))), "set_resolver")

    def sync(self, stream=None):
        """Waits for the stream and raises the first device-detected error."""
        check(self._L.cortado_sync(self._h, _stream(stream)), "device")

    # ------------------------------------------------ reference-shaped operations
    def server_encode(self, d_input, insize, d_output, d_outsize, eb, stream=None):
        check(self._L.cortado_store_encode(self._h, _ptr(d_input), int(insize), float(eb), _ptr(d_output),
                                           _nbytes(d_output), _ptr(d_outsize), _stream(stream)), "server_encode")

    def server_decode(self, d_input, d_output, d_outsize, in_bytes=None, stream=None):
        n = _nbytes(d_input) if in_bytes is None else int(in_bytes)
        check(self._L.cortado_store_decode(self._h, _ptr(d_input), n, _ptr(d_output), _nbytes(d_output),
                                           _ptr(d_outsize), _stream(stream)), "server_decode")

    def s2c_encode(self, d_input, d_output, d_outsize, request_eb, n_bytes, in_bytes=None, stream=None):
        n = _nbytes(d_input) if in_bytes is None else int(in_bytes)
        check(self._L.cortado_init_send(self._h, _ptr(d_input), n, int(n_bytes), float(request_eb), _ptr(d_output),
                                        _nbytes(d_output), _ptr(d_outsize), _stream(stream)), "s2c_encode")

    def client_decode(self, d_input, d_output, d_outsize, in_bytes=None, stream=None):
        n = _nbytes(d_input) if in_bytes is None else int(in_bytes)
        check(self._L.cortado_init_recv(self._h, _ptr(d_input), n, _ptr(d_output), _nbytes(d_output),
                                        _ptr(d_outsize), _stream(stream)), "client_decode")

    def residual_encode(self, d_input, d_output, d_outsize, src_eb, dest_eb, n_bytes, in_bytes=None, stream=None):
        n = _nbytes(d_input) if in_bytes is None else int(in_bytes)
        check(self._L.cortado_resi_send(self._h, _ptr(d_input), n, int(n_bytes), float(src_eb), float(dest_eb),
                                        _ptr(d_output), _nbytes(d_output), _ptr(d_outsize), _stream(stream)),
              "residual_encode")

    def residual_apply(self, d_src, srcsize, d_residual, d_dest, d_destsize, resi_bytes=None, stream=None):
        n = _nbytes(d_residual) if resi_bytes is None else int(resi_bytes)
        check(self._L.cortado_resi_recv(self._h, _ptr(d_src), int(srcsize), _ptr(d_residual), n, _ptr(d_dest),
                                        _nbytes(d_dest), _ptr(d_destsize), _stream(stream)), "residual_apply")

    def s2c_encode_apply(self, d_input, d_output, d_outsize, request_eb, n_bytes, d_client, in_bytes=None,
                         stream=None):
        """init_send fused with the client's init_recv: the init stream into
        d_output and, in the same pass, the client's reconstruction into
        d_client (as client_decode of that stream would write it)."""
        n = _nbytes(d_input) if in_bytes is None else int(in_bytes)
        check(self._L.cortado_init_send_apply(self._h, _ptr(d_input), n, int(n_bytes), float(request_eb),
                                              _ptr(d_output), _nbytes(d_output), _ptr(d_outsize), _ptr(d_client),
                                              _stream(stream)), "s2c_encode_apply")

    def residual_encode_apply(self, d_input, d_output, d_outsize, src_eb, dest_eb, n_bytes, d_client, in_bytes=None,
                              stream=None):
        """resi_send fused with the client's resi_recv: the residual stream
        into d_output, and d_client (the client's floats at src_eb) updated in
        place as residual_apply of that stream would."""
        n = _nbytes(d_input) if in_bytes is None else int(in_bytes)
        check(self._L.cortado_resi_send_apply(self._h, _ptr(d_input), n, int(n_bytes), float(src_eb), float(dest_eb),
                                              _ptr(d_output), _nbytes(d_output), _ptr(d_outsize), _ptr(d_client),
                                              _stream(stream)), "residual_encode_apply")

    def INOA_find_range(self, d_data, size=None, stream=None):
        n = _nbytes(d_data) if size is None else int(size)
        lo, hi = ctypes.c_float(), ctypes.c_float()
        check(self._L.cortado_noa_range(self._h, _ptr(d_data), n, ctypes.byref(lo), ctypes.byref(hi),
                                        _stream(stream)), "INOA_find_range")
        return lo.value, hi.value

    # ------------------------------------------------ NOA bounds on the device
    def INOA_find_range_device(self, d_data, d_minmax=None, size=None, stream=None):
        """The range into a device float32 tensor [min, max] without waiting
        for the device (the NOA entry points below read it there)."""
        if d_minmax is None:
            d_minmax = torch.empty(2, dtype=torch.float32, device=self.device)
        n = _nbytes(d_data) if size is None else int(size)
        check(self._L.cortado_noa_range_device(self._h, _ptr(d_data), n, _ptr(d_minmax), _stream(stream)),
              "INOA_find_range_device")
        return d_minmax

    def server_encode_noa(self, d_input, insize, d_output, d_outsize, d_minmax, eb_noa, stream=None):
        check(self._L.cortado_store_encode_noa(self._h, _ptr(d_input), int(insize), _ptr(d_minmax), float(eb_noa),
                                               _ptr(d_output), _nbytes(d_output), _ptr(d_outsize), _stream(stream)),
              "server_encode_noa")

    def s2c_encode_noa(self, d_input, d_output, d_outsize, d_minmax, request_eb_noa, n_bytes, in_bytes=None,
                       stream=None):
        n = _nbytes(d_input) if in_bytes is None else int(in_bytes)
        check(self._L.cortado_init_send_noa(self._h, _ptr(d_input), n, int(n_bytes), _ptr(d_minmax),
                                            float(request_eb_noa), _ptr(d_output), _nbytes(d_output),
                                            _ptr(d_outsize), _stream(stream)), "s2c_encode_noa")

    def residual_encode_noa(self, d_input, d_output, d_outsize, d_minmax, src_eb_noa, dest_eb_noa, n_bytes,
                            in_bytes=None, stream=None):
        n = _nbytes(d_input) if in_bytes is None else int(in_bytes)
        check(self._L.cortado_resi_send_noa(self._h, _ptr(d_input), n, int(n_bytes), _ptr(d_minmax),
                                            float(src_eb_noa), float(dest_eb_noa), _ptr(d_output),
                                            _nbytes(d_output), _ptr(d_outsize), _stream(stream)),
              "residual_encode_noa")

    def s2c_encode_apply_noa(self, d_input, d_output, d_outsize, d_minmax, request_eb_noa, n_bytes, d_client,
                             in_bytes=None, stream=None):
        """s2c_encode_apply at a NOA request bound of the device range."""
        n = _nbytes(d_input) if in_bytes is None else int(in_bytes)
        check(self._L.cortado_init_send_apply_noa(self._h, _ptr(d_input), n, int(n_bytes), _ptr(d_minmax),
                                                  float(request_eb_noa), _ptr(d_output), _nbytes(d_output),
                                                  _ptr(d_outsize), _ptr(d_client), _stream(stream)),
              "s2c_encode_apply_noa")

    def residual_encode_apply_noa(self, d_input, d_output, d_outsize, d_minmax, src_eb_noa, dest_eb_noa, n_bytes,
                                  d_client, in_bytes=None, stream=None):
        """residual_encode_apply between NOA bounds of the device range."""
        n = _nbytes(d_input) if in_bytes is None else int(in_bytes)
        check(self._L.cortado_resi_send_apply_noa(self._h, _ptr(d_input), n, int(n_bytes), _ptr(d_minmax),
                                                  float(src_eb_noa), float(dest_eb_noa), _ptr(d_output),
                                                  _nbytes(d_output), _ptr(d_outsize), _ptr(d_client),
                                                  _stream(stream)),
              "residual_encode_apply_noa")

    def verify_bound(self, orig, recon, eb_abs, first_bad=None, stream=None):
        """MAXABS_f32 on the device: returns the int64 tensor holding the first
        violating index (or -1 when every value is within eb_abs)."""
        if first_bad is None:
            first_bad = torch.empty(1, dtype=torch.int64, device=self.device)
        check(self._L.cortado_verify_bound(self._h, _ptr(orig), _ptr(recon), _nbytes(orig), float(eb_abs),
                                           _ptr(first_bad), _stream(stream)), "verify_bound")
        return first_bad

    # ------------------------------------------------ batched form
    def batch(self, op: str, items, stream=None):
        """Runs one operation on many streams in a single launch.

        items: sequence of dicts with keys in (tensor), out (tensor), out_size
        (int64 tensor slice), n_bytes, and as the operation needs eb1, eb2,
        src (tensor), in_bytes (defaults to in's size)."""
        arr = (_native.Item * len(items))()
        for i, it in enumerate(items):
            x = arr[i]
            x.d_in = _ptr(it["in"])
            x.in_bytes = int(it.get("in_bytes", _nbytes(it["in"])))
            x.n_bytes = int(it["n_bytes"])
            x.eb1 = float(it.get("eb1", 0.0))
            x.eb2 = float(it.get("eb2", 0.0))
            x.d_src = _ptr(it.get("src"))
            x.d_out = _ptr(it["out"])
            x.out_capacity = int(it.get("out_capacity", _nbytes(it["out"])))
            x.d_outsize = _ptr(it["out_size"])
        check(self._L.cortado_batch(self._h, _native.OPS[op], ctypes.cast(arr, ctypes.c_void_p), len(items),
                                    _stream(stream)), "batch " + op)

    # ------------------------------------------------ convenience forms
    def _empty_stream(self, n_bytes):
        return torch.empty(max_stream_bytes(n_bytes), dtype=torch.uint8, device=self.device)

    def _trim(self, buf, size):
        self.sync()
        return buf[: int(size.item())]

    def store(self, x: torch.Tensor, eb_abs: float) -> torch.Tensor:
        x = x.contiguous()
        out = self._empty_stream(_nbytes(x))
        size = torch.empty(1, dtype=torch.int64, device=self.device)
        self.server_encode(x, _nbytes(x), out, size, eb_abs)
        return self._trim(out, size)

    def store_decode(self, stored: torch.Tensor, n_bytes: int | None = None) -> torch.Tensor:
        n = n_bytes if n_bytes is not None else stream_orig_bytes(stored)
        out = torch.empty(max(n, 4) // 4, dtype=torch.float32, device=self.device)
        size = torch.empty(1, dtype=torch.int64, device=self.device)
        self.server_decode(stored, out, size)
        self.sync()
        return out[: n // 4]

    def init_send(self, stored: torch.Tensor, request_eb_abs: float, n_bytes: int | None = None) -> torch.Tensor:
        n = n_bytes if n_bytes is not None else stream_orig_bytes(stored)
        out = self._empty_stream(n)
        size = torch.empty(1, dtype=torch.int64, device=self.device)
        self.s2c_encode(stored, out, size, request_eb_abs, n)
        return self._trim(out, size)

    def init_recv(self, init: torch.Tensor, n_bytes: int | None = None) -> torch.Tensor:
        n = n_bytes if n_bytes is not None else stream_orig_bytes(init)
        out = torch.empty(max(n, 4) // 4, dtype=torch.float32, device=self.device)
        size = torch.empty(1, dtype=torch.int64, device=self.device)
        self.client_decode(init, out, size)
        self.sync()
        return out[: n // 4]

    def resi_send(self, stored: torch.Tensor, src_eb_abs: float, dst_eb_abs: float,
                  n_bytes: int | None = None) -> torch.Tensor:
        n = n_bytes if n_bytes is not None else stream_orig_bytes(stored)
        out = self._empty_stream(n)
        size = torch.empty(1, dtype=torch.int64, device=self.device)
        self.residual_encode(stored, out, size, src_eb_abs, dst_eb_abs, n)
        return self._trim(out, size)

    def resi_recv(self, src: torch.Tensor, resi: torch.Tensor) -> torch.Tensor:
        src = src.contiguous()
        out = torch.empty_like(src, dtype=torch.float32)
        size = torch.empty(1, dtype=torch.int64, device=self.device)
        self.residual_apply(src, _nbytes(src), resi, out, size)
        self.sync()
        return out


def stream_orig_bytes(stream: torch.Tensor) -> int:
    """Original size from a stream header (reads 8 bytes to the host)."""
    return int(stream[:8].cpu().view(torch.int64).item())
