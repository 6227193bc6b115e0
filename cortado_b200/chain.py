"""Progressive refinement chain captured as one CUDA graph.

A field is stored once at several bounds.  Then the client's whole request
sequence -- init at a coarse bound, then residual steps to ever finer bounds,
each applied client-side on the device -- runs as a single graph launch:

    init_send -> init_recv -> verify
    resi_send -> resi_recv -> verify      (one pair per refinement step)

Each step reads the stored stream the reference's CLIs would choose (the
first stored bound not above the step's target, src/cortado_init.cu:298-304,
src/cortado_resi.cu:334-348).  It checks its reconstruction against the
original with the device bound verifier (MAXABS_f32 rules).  All buffers are
allocated before capture and the lookback epoch lives in device memory, so
replays are independent.
"""
from __future__ import annotations

import torch

from . import storage
from .ops import Codec, max_stream_bytes


class ProgressiveChain:
    def __init__(self, codec: Codec, x: torch.Tensor, store_bounds_abs, init_eb_abs, step_bounds_abs):
        self.c = codec
        self.x = x.contiguous().view(-1)
        self.n = self.x.numel() * 4
        dev = self.x.device
        self.store_bounds = sorted((float(e) for e in store_bounds_abs), reverse=True)
        self.bounds = [float(init_eb_abs)] + [float(e) for e in step_bounds_abs]
        cap = max_stream_bytes(self.n)
        self.sizes = torch.zeros(2 * len(self.bounds) + len(self.store_bounds), dtype=torch.int64, device=dev)
        # stored streams: produced once, outside the graph
        self.stored = []
        for i, eb in enumerate(self.store_bounds):
            buf = torch.empty(cap, dtype=torch.uint8, device=dev)
            codec.server_encode(self.x, self.n, buf, self.sizes[i:i + 1], eb)
            self.stored.append(buf)
        codec.sync()
        self.stored_bytes = [int(v) for v in self.sizes[: len(self.store_bounds)].tolist()]
        k = len(self.store_bounds)
        self.streams = [torch.empty(cap, dtype=torch.uint8, device=dev) for _ in self.bounds]
        self.recon = [torch.empty_like(self.x) for _ in self.bounds]
        self.first_bad = torch.empty(len(self.bounds), dtype=torch.int64, device=dev)
        self.stream_sizes = self.sizes[k: k + len(self.bounds)]
        self.recon_sizes = self.sizes[k + len(self.bounds):]
        self.sel = []
        for j, dst in enumerate(self.bounds):
            i = storage.select_stored([storage.f32(e) for e in self.store_bounds], dst)
            if i < 0:
                raise ValueError(f"bound {dst} is tighter than every stored bound")
            self.sel.append(i)
        self.graph = None

    def _enqueue(self, s):
        c = self.c
        b = self.bounds
        i = self.sel[0]
        c.s2c_encode(self.stored[i], self.streams[0], self.stream_sizes[0:1], b[0], self.n,
                     in_bytes=self.stored_bytes[i], stream=s)
        c.client_decode(self.streams[0], self.recon[0], self.recon_sizes[0:1], stream=s)
        c.verify_bound(self.x, self.recon[0], b[0], self.first_bad[0:1], stream=s)
        for j in range(1, len(b)):
            i = self.sel[j]
            c.residual_encode(self.stored[i], self.streams[j], self.stream_sizes[j:j + 1], b[j - 1], b[j], self.n,
                              in_bytes=self.stored_bytes[i], stream=s)
            c.residual_apply(self.recon[j - 1], self.n, self.streams[j], self.recon[j], self.recon_sizes[j:j + 1],
                             stream=s)
            c.verify_bound(self.x, self.recon[j], b[j], self.first_bad[j:j + 1], stream=s)

    def run_eager(self, stream=None):
        s = stream or torch.cuda.current_stream()
        self._enqueue(s)

    def capture(self):
        """Captures the chain (run it eagerly once first, so the context's
        scratch is already large enough and nothing allocates under capture)."""
        self.run_eager()
        self.c.sync()
        s = torch.cuda.Stream(self.x.device)
        s.wait_stream(torch.cuda.current_stream())
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=s):
            self._enqueue(s)
        torch.cuda.current_stream().wait_stream(s)
        return self.graph

    def replay(self):
        self.graph.replay()

    def launches(self) -> int:
        return 3 + 3 * (len(self.bounds) - 1)
