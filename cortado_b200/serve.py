"""Continuous-batching request server for progressive retrieval.

The server keeps every field's stored streams (one per stored bound) and every
client's current reconstruction resident in HBM.  Requests:

* ``init``  (client, field, bound): init_send from the stored stream the
  reference's CLI would pick, then init_recv into the client's reconstruction;
* ``resi``  (client, field, bound): resi_send from the client's current bound
  to the requested one, then resi_recv applied to the client's
  reconstruction in place.

Requests arrive over time (``Request.arrival`` in seconds from the start).
Each loop iteration admits arrived requests, in arrival order, up to
``max_batch`` per batch.  Admission needs a free slot (``max_inflight``),
device memory under ``mem_cap_bytes`` for its output stream, and no earlier
request of the same client on the same field still running or waiting (a
client's steps are ordered); a request held back for that reason does not hold
back other clients' requests.  The admitted requests are grouped by operation
and run as batched launches (``cortado_batch``: one persistent launch per
operation for the whole group) on one of ``n_streams`` CUDA streams.
Admission does not wait for earlier batches: a new batch starts on the next
stream while others are still on the GPU (several batches in flight keep the
GPU busy while the host assembles the next one), and completions are polled
with CUDA events.  A request's
latency is its completion time (the host clock when its batch's event is seen
complete) minus its arrival.

``run_plain`` serves the same trace with the plain per-request pipeline (one
operation per launch, synchronized after each request) for comparison.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import storage
from .ops import Codec, max_stream_bytes


@dataclass
class Request:
    rid: int
    kind: str          # "init" or "resi"
    client: int
    field: str
    bound: float       # absolute destination bound
    arrival: float     # seconds from the start of the run
    done: float = -1.0
    out_bytes: int = 0


@dataclass
class Field:
    name: str
    x: torch.Tensor                 # original floats (device), kept for verification only
    store_bounds: list              # absolute, descending
    stored: list = field(default_factory=list)
    stored_bytes: list = field(default_factory=list)

    @property
    def n_bytes(self):
        return self.x.numel() * 4


class Server:
    def __init__(self, device=0, mem_cap_bytes=120 * 10**9, max_inflight=64, n_streams=3, max_batch=16):
        self.dev = torch.device("cuda", device)
        self.codecs = [Codec(device) for _ in range(n_streams)]
        self.streams = [torch.cuda.Stream(self.dev) for _ in range(n_streams)]
        self.mem_cap = mem_cap_bytes
        self.max_inflight = max_inflight
        self.max_batch = max_batch
        self.fields: dict[str, Field] = {}
        self.clients: dict[tuple, dict] = {}   # (client, field) -> {"recon": tensor, "bound": float}
        self.mem_used = 0
        # Output stream buffers, per field (each field's capacity is fixed),
        # reused once the batch that held one is seen complete: after a
        # warm-up the loop allocates no device memory.  (Allocating per request
        # through the caching allocator, across several streams, sometimes
        # fell back to a fresh cudaMalloc, which stalls the device.)
        self._free_out: dict[str, list[torch.Tensor]] = {}

    # ---------------------------------------------------------------- storage
    def add_field(self, name, x, store_bounds_abs):
        f = Field(name, x.contiguous().view(-1), sorted((float(e) for e in store_bounds_abs), reverse=True))
        c = self.codecs[0]
        for eb in f.store_bounds:
            s = c.store(f.x, eb)
            f.stored.append(s)
            f.stored_bytes.append(s.numel())
            self.mem_used += s.numel()
        self.fields[name] = f

    def _recon(self, client, fname):
        key = (client, fname)
        st = self.clients.get(key)
        if st is None:
            f = self.fields[fname]
            st = {"recon": torch.empty(f.x.numel(), dtype=torch.float32, device=self.dev), "bound": None}
            self.clients[key] = st
            self.mem_used += f.n_bytes
        return st

    def _out_buffer(self, f: Field) -> torch.Tensor:
        free = self._free_out.get(f.name)
        if free:
            return free.pop()
        return torch.empty(max_stream_bytes(f.n_bytes), dtype=torch.uint8, device=self.dev)

    def _stored_for(self, f: Field, bound):
        i = storage.select_stored([storage.f32(e) for e in f.store_bounds], bound)
        if i < 0:
            raise ValueError(f"bound {bound} is tighter than every stored bound of {f.name}")
        return f.stored[i]

    # ---------------------------------------------------------------- batches
    def _launch(self, k, reqs):
        """Enqueues one batch (any mix of init and resi requests) on stream k."""
        codec, s = self.codecs[k], self.streams[k]
        inits = [r for r in reqs if r.kind == "init"]
        resis = [r for r in reqs if r.kind == "resi"]
        # Everything this batch allocates is allocated on its own stream, so the
        # caching allocator orders the memory with the batch's launches.
        with torch.cuda.stream(s):
            sizes = torch.empty(max(1, len(reqs)) * 2, dtype=torch.int64, device=self.dev)
        outs = {}
        j = 0
        items_send, items_recv = [], []
        for r in inits:
            f = self.fields[r.field]
            st = self._recon(r.client, r.field)
            out = self._out_buffer(f)
            outs[r.rid] = out
            items_send.append(dict(**{"in": self._stored_for(f, r.bound)}, out=out, out_size=sizes[j:j + 1],
                                   n_bytes=f.n_bytes, eb1=r.bound))
            items_recv.append(dict(**{"in": out}, out=st["recon"], out_size=sizes[j + 1:j + 2], n_bytes=f.n_bytes))
            st["bound"] = r.bound
            j += 2
        with torch.cuda.stream(s):
            if items_send:
                codec.batch("init_send", items_send, stream=s)
                codec.batch("init_recv", items_recv, stream=s)
        items_send, items_recv = [], []
        for r in resis:
            f = self.fields[r.field]
            st = self._recon(r.client, r.field)
            if st["bound"] is None:
                raise ValueError(f"request {r.rid}: residual before init")
            out = self._out_buffer(f)
            outs[r.rid] = out
            items_send.append(dict(**{"in": self._stored_for(f, r.bound)}, out=out, out_size=sizes[j:j + 1],
                                   n_bytes=f.n_bytes, eb1=st["bound"], eb2=r.bound))
            items_recv.append(dict(**{"in": out}, src=st["recon"], out=st["recon"], out_size=sizes[j + 1:j + 2],
                                   n_bytes=f.n_bytes))
            st["bound"] = r.bound
            j += 2
        with torch.cuda.stream(s):
            if items_send:
                codec.batch("resi_send", items_send, stream=s)
                codec.batch("resi_recv", items_recv, stream=s)
        ev = torch.cuda.Event()
        ev.record(s)
        return ev, outs, sizes

    # ---------------------------------------------------------------- loops
    def run(self, requests: list[Request], keep_outputs=False):
        """Serves the trace with continuous batching; returns stats."""
        pending = sorted(requests, key=lambda r: r.arrival)
        inflight = []          # (event, reqs, outs, sizes, bytes, stream index)
        waiting = []           # arrived, not yet admitted, in arrival order
        busy_clients = set()
        outputs = {}
        t0 = time.perf_counter()
        k = 0
        i = 0
        while i < len(pending) or waiting or inflight:
            now = time.perf_counter() - t0
            # completions
            still = []
            for item in inflight:
                ev, reqs, outs, sizes, nbytes, _ = item
                if ev.query():
                    tdone = time.perf_counter() - t0
                    for r in reqs:
                        r.done = tdone
                        busy_clients.discard((r.client, r.field))
                    for r in reqs:
                        if keep_outputs:  # handed to the caller, not reused
                            outputs[r.rid] = outs[r.rid]
                        else:
                            self._free_out.setdefault(r.field, []).append(outs[r.rid])
                    self.mem_used -= nbytes
                else:
                    still.append(item)
            inflight = still
            # admission: in arrival order, except that a request whose client
            # (on that field) has an earlier step running or waiting is passed
            # over, together with that client's later requests
            while i < len(pending) and pending[i].arrival <= now:
                waiting.append(pending[i])
                i += 1
            batch, nbytes = [], 0
            room = min(self.max_batch, self.max_inflight - sum(len(x[1]) for x in inflight))
            if room > 0 and waiting:
                held, keep = set(), []
                for j, r in enumerate(waiting):
                    if len(batch) >= room:
                        keep.extend(waiting[j:])
                        break
                    key = (r.client, r.field)
                    if key in busy_clients or key in held:
                        held.add(key)
                        keep.append(r)
                        continue
                    need = max_stream_bytes(self.fields[r.field].n_bytes)
                    if self.mem_used + nbytes + need > self.mem_cap:
                        keep.extend(waiting[j:])
                        break
                    batch.append(r)
                    busy_clients.add(key)
                    nbytes += need
                waiting = keep
            if batch:
                self.mem_used += nbytes
                ev, outs, sizes = self._launch(k, batch)
                inflight.append((ev, batch, outs, sizes, nbytes, k))
                k = (k + 1) % len(self.streams)
            elif inflight:
                time.sleep(20e-6)
            elif waiting:
                raise RuntimeError(f"request {waiting[0].rid} needs more than the {self.mem_cap}-byte memory cap")
            elif i < len(pending):
                time.sleep(max(0.0, min(1e-3, pending[i].arrival - (time.perf_counter() - t0))))
        for c, s in zip(self.codecs, self.streams):
            c.sync(s)
        wall = time.perf_counter() - t0
        return self._stats(requests, wall), outputs

    def run_plain(self, requests: list[Request], keep_outputs=False):
        """The plain per-request pipeline: requests in arrival order, each as
        its own send and receive call (the reference-shaped single-stream entry
        points, decoding straight into the client's reconstruction),
        synchronized after every request."""
        pending = sorted(requests, key=lambda r: r.arrival)
        codec, s = self.codecs[0], self.streams[0]
        outputs = {}
        with torch.cuda.stream(s):
            sizes = torch.empty(2, dtype=torch.int64, device=self.dev)
        t0 = time.perf_counter()
        for r in pending:
            now = time.perf_counter() - t0
            if r.arrival > now:
                time.sleep(r.arrival - now)
            f = self.fields[r.field]
            st = self._recon(r.client, r.field)
            stored = self._stored_for(f, r.bound)
            with torch.cuda.stream(s):
                out = torch.empty(max_stream_bytes(f.n_bytes), dtype=torch.uint8, device=self.dev)
                if r.kind == "init":
                    codec.s2c_encode(stored, out, sizes[0:1], r.bound, f.n_bytes, stream=s)
                    codec.client_decode(out, st["recon"], sizes[1:2], stream=s)
                else:
                    codec.residual_encode(stored, out, sizes[0:1], st["bound"], r.bound, f.n_bytes, stream=s)
                    codec.residual_apply(st["recon"], f.n_bytes, out, st["recon"], sizes[1:2], stream=s)
                st["bound"] = r.bound
            codec.sync(s)
            r.done = time.perf_counter() - t0
            if keep_outputs:
                outputs[r.rid] = out
        wall = time.perf_counter() - t0
        return self._stats(requests, wall), outputs

    def _stats(self, requests, wall):
        lat = np.array([r.done - r.arrival for r in requests if r.done >= 0])
        orig = sum(self.fields[r.field].n_bytes for r in requests if r.done >= 0)
        return {"requests": len(lat), "wall_s": wall, "orig_GBps": orig * 1e-9 / wall if wall > 0 else None,
                "p50_ms": float(np.percentile(lat, 50) * 1e3) if lat.size else None,
                "p99_ms": float(np.percentile(lat, 99) * 1e3) if lat.size else None}

    def prepare(self, requests: list[Request]):
        """Allocates the reconstruction of every (client, field) the requests
        touch, as a server does when a client opens a field, and sizes every
        context's scratch for the largest batch (max_batch requests on the
        largest field), so that serving itself allocates only output streams."""
        for r in requests:
            self._recon(r.client, r.field)
        if self.fields:
            chunks = max(-(-f.n_bytes // 16384) for f in self.fields.values())
            for c in self.codecs:
                c.reserve(self.max_batch * chunks, self.max_batch)
        torch.cuda.synchronize(self.dev)

    def reset_clients(self, free=True):
        """Forgets every client's progress; free=False keeps the buffers."""
        if not free:
            for st in self.clients.values():
                st["bound"] = None
            return
        for (c, fname), st in self.clients.items():
            self.mem_used -= self.fields[fname].n_bytes
        self.clients.clear()

    def close(self):
        for c in self.codecs:
            c.close()


def poisson_trace(rng: np.random.Generator, fields_: dict, n_requests: int, rate_hz: float, n_clients: int,
                  ranges: dict):
    """60% init requests (bound log-uniform in [1e-3, 1e-1] of the field's
    range) and 40% residual requests (1 to 3 decades finer than the client's
    current bound), Poisson arrivals at rate_hz.  A client's first request on
    a field is always an init.  ``ranges`` maps field -> value range (NOA)."""
    reqs, t = [], 0.0
    cur = {}
    names = sorted(fields_)
    for rid in range(n_requests):
        t += rng.exponential(1.0 / rate_hz)
        client = int(rng.integers(n_clients))
        fname = names[int(rng.integers(len(names)))]
        key = (client, fname)
        if key not in cur or rng.random() < 0.6:
            noa = float(10 ** rng.uniform(-3, -1))
            kind = "init"
        else:
            noa = cur[key] * float(10 ** -rng.uniform(1, 3))
            kind = "resi"
        noa = max(noa, 1e-6)
        if kind == "resi" and noa >= cur[key]:
            kind = "init"
        cur[key] = noa
        reqs.append(Request(rid, kind, client, fname, float(storage.noa_scale(noa, ranges[fname])), t))
    return reqs
