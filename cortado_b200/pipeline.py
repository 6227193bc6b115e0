"""Host <-> device pipelines: many host-resident fields through the device
path with the copies overlapped.

The reference's drivers handle one field at a time: copy it to the device,
run the operation, copy the result back (src/cortado_store.cu:189-203,
283-286), each step waiting for the previous one.  Here two device slots
alternate.  Item i+1's host->device copy runs on a load stream while item i
runs on its slot's compute stream.  Item i's device->host copy runs on a store
stream after it, overlapping item i+1's compute.  The two copy directions use
independent copy engines.  Events order only the reuse of a slot's buffers.

``Pipeline`` is the scheduler: the caller supplies what to copy in, what to run
and what to copy out per item.  ``StorePipeline`` uses it to store host fields
at several bounds and return the streams in host memory.
"""
from __future__ import annotations

from typing import Callable, Sequence

import torch

from .ops import Codec, max_stream_bytes


class Pipeline:
    """Two-slot host<->device pipeline over n items.

    load(i, slot, stream)  enqueues item i's host->device copies on `stream`;
    run(i, slot, stream)   enqueues item i's device work on `stream` (the
                           slot's compute stream; it may block the host, e.g.
                           to read a NOA range);
    store(i, slot, stream) enqueues item i's device->host copies on `stream`.

    Each callable enqueues only on the stream it is given; run() may read the
    slot's inputs only, and store() the slot's outputs only.  `slots` holds
    two caller objects with a `stream` attribute (the compute stream).
    """

    def __init__(self, device, slots: Sequence, load: Callable, run: Callable, store: Callable):
        if len(slots) != 2:
            raise ValueError("a pipeline has two slots")
        self.dev = torch.device(device)
        self.slots = list(slots)
        self.load, self.run, self.store = load, run, store
        self.s_in = torch.cuda.Stream(self.dev)
        self.s_out = torch.cuda.Stream(self.dev)
        self.ev_in = [torch.cuda.Event() for _ in slots]    # the slot's inputs have arrived
        self.ev_done = [torch.cuda.Event() for _ in slots]  # the slot's device work has finished
        self.ev_out = [torch.cuda.Event() for _ in slots]   # the slot's outputs have been copied out
        for k, sl in enumerate(self.slots):
            self.ev_done[k].record(sl.stream)
            self.ev_out[k].record(sl.stream)

    def _load(self, i):
        k = i % 2
        self.s_in.wait_event(self.ev_done[k])  # the slot's previous item has read its inputs
        with torch.cuda.stream(self.s_in):
            self.load(i, self.slots[k], self.s_in)
        self.ev_in[k].record(self.s_in)

    def _run_store(self, i):
        k = i % 2
        sl = self.slots[k]
        sl.stream.wait_event(self.ev_in[k])
        sl.stream.wait_event(self.ev_out[k])  # the slot's previous outputs have been copied out
        with torch.cuda.stream(sl.stream):
            self.run(i, sl, sl.stream)
        self.ev_done[k].record(sl.stream)
        self.s_out.wait_event(self.ev_done[k])
        with torch.cuda.stream(self.s_out):
            self.store(i, sl, self.s_out)
        self.ev_out[k].record(self.s_out)

    def __call__(self, n_items: int):
        """Enqueues all n items; returns without waiting (see sync())."""
        if n_items <= 0:
            return
        self._load(0)
        for i in range(n_items):
            if i + 1 < n_items:
                self._load(i + 1)
            self._run_store(i)

    def sync(self):
        self.s_out.synchronize()
        for sl in self.slots:
            sl.stream.synchronize()


class _StoreSlot:
    def __init__(self, device, max_bytes: int, n_bounds: int):
        self.codec = Codec(device)
        self.stream = torch.cuda.Stream(device)
        self.x = torch.empty(max_bytes // 4, dtype=torch.float32, device=device)
        cap = max_stream_bytes(max_bytes)
        self.out = [torch.empty(cap, dtype=torch.uint8, device=device) for _ in range(n_bounds)]
        self.sizes = torch.zeros(n_bounds, dtype=torch.int64, device=device)
        self.h_sizes = torch.zeros(n_bounds, dtype=torch.int64).pin_memory()


class StorePipeline:
    """Stores host float32 fields at several absolute bounds each (the store
    operation, d_server_encode, once per bound) with overlapped copies.

    run(fields, bounds) takes CPU float32 tensors (pinned ones are copied
    straight from; others are staged through pinned memory once) and one list
    of absolute bounds per field (all lists of the same length).  It returns,
    per field, the stored streams as CPU uint8 tensors, byte-identical to
    Codec.store.  A stream's size is known only once its encode has finished,
    so each item's copies out are issued after its device work completes,
    while the next item's copy in and encode are already queued.
    """

    def __init__(self, device, max_bytes: int, n_bounds: int):
        self.dev = torch.device(device)
        if max_bytes <= 0 or max_bytes % 4:
            raise ValueError("max_bytes must be a positive multiple of 4")
        self.max_bytes = max_bytes
        self.n_bounds = n_bounds
        self.slots = [_StoreSlot(self.dev, max_bytes, n_bounds) for _ in range(2)]

    def close(self):
        for sl in self.slots:
            sl.codec.close()

    def run(self, fields: Sequence[torch.Tensor], bounds: Sequence[Sequence[float]]) -> list[list[torch.Tensor]]:
        if len(fields) != len(bounds):
            raise ValueError("one list of bounds per field")
        hosts = []
        for f in fields:
            f = f.reshape(-1)
            if f.dtype != torch.float32 or f.device.type != "cpu":
                raise ValueError("fields must be CPU float32 tensors")
            if f.numel() * 4 > self.max_bytes or f.numel() == 0:
                raise ValueError(f"field of {f.numel() * 4} bytes outside 1..{self.max_bytes}")
            hosts.append(f.contiguous() if f.is_pinned() else f.contiguous().pin_memory())
        for b in bounds:
            if len(b) != self.n_bounds:
                raise ValueError(f"each field needs {self.n_bounds} bounds")
        results: list[list[torch.Tensor]] = [[] for _ in fields]

        def load(i, sl, s):
            n = hosts[i].numel()
            sl.x[:n].copy_(hosts[i], non_blocking=True)

        def run(i, sl, s):
            n = hosts[i].numel()
            for j, eb in enumerate(bounds[i]):
                sl.codec.server_encode(sl.x[:n], n * 4, sl.out[j], sl.sizes[j:j + 1], float(eb), stream=s)
            sl.h_sizes.copy_(sl.sizes, non_blocking=True)

        def store(i, sl, s):
            # `s` waits for this item's device work, which ends with the copy
            # of its sizes; wait for it on the host to size the copies out
            s.synchronize()
            sl.codec.sync(sl.stream)
            for j in range(self.n_bounds):
                nb = int(sl.h_sizes[j])
                h = torch.empty(nb, dtype=torch.uint8, pin_memory=True)
                h.copy_(sl.out[j][:nb], non_blocking=True)
                results[i].append(h)

        pipe = Pipeline(self.dev, self.slots, load, run, store)
        pipe(len(hosts))
        pipe.sync()
        for sl in self.slots:
            sl.codec.sync(sl.stream)
        return results
