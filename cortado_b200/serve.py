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
operation for the whole group) on one of ``n_streams`` CUDA streams.  Each
launch is a send fused with the client's receive (init_send_apply,
resi_send_apply): it writes the stream that goes to the client and, in the
same pass, the client's resident reconstruction, exactly as a separate
receive of that stream would.
Admission does not wait for earlier batches: a new batch starts on the next
stream while others are still on the GPU (several batches in flight keep the
GPU busy while the host assembles the next one), and completions are polled
with CUDA events.  A request's
latency is its completion time (the host clock when its batch's event is seen
complete) minus its arrival.

Device memory is admitted against ``mem_cap_bytes``: resident stored streams,
resident client reconstructions and output stream buffers (in flight or
pooled for reuse) are counted.  A request's admission reserves its output
buffer, its client's reconstruction (when that client has none resident)
and its field's stored streams (when they are not resident).  When a request
does not fit, idle state is spilled to host files until it does, least
recently used first: pooled output buffers are freed, then idle clients'
reconstructions are written as raw float32 files (the reference's
decoded-file format, which its resi_recv reads back as the client's source,
src/cortado_resi.cu:393-410), then idle fields' stored streams as a server
storage directory (``<field>.stor.NN`` + ``.stor.meta``,
include/util.h:70-135).  "Idle" means that no admitted, unfinished request
uses it.  Spilled state is read back when a request needs it.  Only a
request larger than the cap by itself is an error.

``run_plain`` serves the same trace with the plain per-request pipeline (one
operation per launch, synchronized after each request) for comparison.
"""
from __future__ import annotations

import contextlib
import os
import tempfile
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
    stored: list = field(default_factory=list)        # device streams (empty while spilled)
    stored_bytes: list = field(default_factory=list)
    vrange: float = 0.0             # max - min of the original (written to .stor.meta)
    spilled: str | None = None      # storage directory holding the streams while not resident
    last_use: int = 0

    @property
    def n_bytes(self):
        return self.x.numel() * 4

    @property
    def stored_total(self):
        return sum(self.stored_bytes)


class Server:
    def __init__(self, device=0, mem_cap_bytes=120 * 10**9, max_inflight=64, n_streams=3, max_batch=16,
                 spill_dir: str | None = None, max_batches: int | None = None):
        self.dev = torch.device("cuda", device)
        self.codecs = [Codec(device) for _ in range(n_streams)]
        self.streams = [torch.cuda.Stream(self.dev) for _ in range(n_streams)]
        self.mem_cap = mem_cap_bytes
        self.max_inflight = max_inflight
        self.max_batch = max_batch
        # batches in flight at most (None: one per stream; 0: no limit besides
        # max_inflight requests).  While that many run, arrivals gather into
        # the next batch: at 8000 requests/s the bench's trace then runs as 35
        # batches instead of about 100, at the same rate.
        self.max_batches = n_streams if max_batches is None else max_batches
        self.fields: dict[str, Field] = {}
        # (client, field) -> {"recon": tensor or None (not resident), "bound": float or None,
        #                     "spilled": host file or None, "last_use": int}
        self.clients: dict[tuple, dict] = {}
        self.mem_used = 0
        self.spill_dir = spill_dir
        self.spills = 0
        self.reloads = 0
        self._tick = 0
        # Output stream buffers, per field (each field's capacity is fixed),
        # reused once the batch that held one is seen complete: after a
        # warm-up the loop allocates no device memory.  (Allocating per request
        # through the caching allocator, across several streams, sometimes
        # fell back to a fresh cudaMalloc, which stalls the device.)  Pooled
        # buffers count against the memory cap until they are freed.
        self._free_out: dict[str, list[torch.Tensor]] = {}
        self._timeline = []

    # ---------------------------------------------------------------- storage
    def add_field(self, name, x, store_bounds_abs, vrange=None):
        f = Field(name, x.contiguous().view(-1), sorted((float(e) for e in store_bounds_abs), reverse=True))
        f.vrange = float(vrange) if vrange is not None else float(f.x.max() - f.x.min())
        c = self.codecs[0]
        for eb in f.store_bounds:
            s = c.store(f.x, eb)
            f.stored.append(s)
            f.stored_bytes.append(s.numel())
            self.mem_used += s.numel()
        self.fields[name] = f
        self._make_room(0, protect_fields={name}, protect_clients=set())

    def _on(self, stream):
        """Context that makes `stream` current (no-op for a host device)."""
        if self.dev.type != "cuda":
            return contextlib.nullcontext()
        return torch.cuda.stream(stream or torch.cuda.current_stream(self.dev))

    def _spill_root(self) -> str:
        if self.spill_dir is None:
            self.spill_dir = tempfile.mkdtemp(prefix="cortado_spill_")
        os.makedirs(self.spill_dir, exist_ok=True)
        return self.spill_dir

    def _spill_field(self, f: Field):
        """Writes the field's stored streams as a storage directory and frees
        them on the device."""
        d = os.path.join(self._spill_root(), "fields", f.name)
        storage.write_storage(d, f.name, [t.cpu().numpy() for t in f.stored], f.store_bounds, f.vrange)
        f.stored = []
        f.spilled = d
        self.mem_used -= f.stored_total
        self.spills += 1

    def _reload_field(self, f: Field, stream):
        meta = storage.read_storage_meta(f.spilled)
        assert [float(e) for e in meta.ebs] == [float(np.float32(e)) for e in f.store_bounds]
        with self._on(stream):
            for i, nb in enumerate(f.stored_bytes):
                h = np.fromfile(os.path.join(f.spilled, storage.stor_name(f.name, i)), dtype=np.uint8)
                assert h.size == nb
                f.stored.append(torch.from_numpy(h).to(self.dev))
        f.spilled = None
        self.mem_used += f.stored_total
        self.reloads += 1

    def _spill_client(self, key, st):
        f = self.fields[key[1]]
        if st["bound"] is not None:  # a client with progress: its floats are its state
            path = os.path.join(self._spill_root(), "clients", f"c{key[0]}_{key[1]}.f32")
            os.makedirs(os.path.dirname(path), exist_ok=True)
            st["recon"].cpu().numpy().tofile(path)
            st["spilled"] = path
        st["recon"] = None
        self.mem_used -= f.n_bytes
        self.spills += 1

    def _recon(self, client, fname, stream=None, reload=True):
        """The client's reconstruction of a field, allocated (and counted) if
        it has none resident; reload=True reads a spilled one back."""
        key = (client, fname)
        st = self.clients.get(key)
        if st is None:
            st = {"recon": None, "bound": None, "spilled": None, "last_use": 0}
            self.clients[key] = st
        if st["recon"] is None:
            f = self.fields[fname]
            with self._on(stream):
                st["recon"] = torch.empty(f.x.numel(), dtype=torch.float32, device=self.dev)
                if reload and st["spilled"]:
                    st["recon"].copy_(torch.from_numpy(np.fromfile(st["spilled"], dtype=np.float32)))
                    self.reloads += 1
            st["spilled"] = None
            self.mem_used += f.n_bytes
        return st

    def _resident(self, key) -> bool:
        st = self.clients.get(key)
        return st is not None and st["recon"] is not None

    def _out_buffer(self, f: Field) -> torch.Tensor:
        free = self._free_out.get(f.name)
        if free:
            return free.pop()
        self.mem_used += max_stream_bytes(f.n_bytes)
        return torch.empty(max_stream_bytes(f.n_bytes), dtype=torch.uint8, device=self.dev)

    def _stored_for(self, f: Field, bound):
        i = storage.select_stored([storage.f32(e) for e in f.store_bounds], bound)
        if i < 0:
            raise ValueError(f"bound {bound} is tighter than every stored bound of {f.name}")
        return f.stored[i]

    # ---------------------------------------------------------------- memory
    def _make_room(self, need, protect_fields, protect_clients, keep_pool=None) -> bool:
        """Frees idle state until mem_used + need fits the cap: pooled output
        buffers (all but keep_pool[field] of each field's), then idle clients'
        reconstructions, then idle fields' stored streams, least recently used
        first.  Returns whether it fits."""
        keep_pool = keep_pool or {}
        if self.mem_used + need <= self.mem_cap:
            return True
        for name, pool in self._free_out.items():
            keep = keep_pool.get(name, 0)
            while len(pool) > keep and self.mem_used + need > self.mem_cap:
                pool.pop()
                self.mem_used -= max_stream_bytes(self.fields[name].n_bytes)
        idle = sorted(((st["last_use"], key) for key, st in self.clients.items()
                       if st["recon"] is not None and key not in protect_clients), key=lambda t: t[0])
        for _, key in idle:
            if self.mem_used + need <= self.mem_cap:
                break
            self._spill_client(key, self.clients[key])
        idle_f = sorted(((f.last_use, f.name) for f in self.fields.values()
                         if f.spilled is None and f.name not in protect_fields), key=lambda t: t[0])
        for _, name in idle_f:
            if self.mem_used + need <= self.mem_cap:
                break
            self._spill_field(self.fields[name])
        return self.mem_used + need <= self.mem_cap

    def _materialize(self, reqs, stream):
        """Makes the state the requests use resident (reads spilled fields and
        reconstructions back on `stream`; an init's reconstruction is only
        allocated, its old contents are not needed)."""
        for r in reqs:
            f = self.fields[r.field]
            if f.spilled is not None:
                self._reload_field(f, stream)
            self._recon(r.client, r.field, stream, reload=r.kind == "resi")

    # ---------------------------------------------------------------- batches
    def _launch(self, k, reqs):
        """Enqueues one batch (any mix of init and resi requests) on stream k:
        both item lists are built first, so the batch's two launches follow
        each other on the stream with no host work between them."""
        codec, s = self.codecs[k], self.streams[k]
        inits = [r for r in reqs if r.kind == "init"]
        resis = [r for r in reqs if r.kind == "resi"]
        # Everything this batch allocates is allocated on its own stream, so the
        # caching allocator orders the memory with the batch's launches.
        with torch.cuda.stream(s):
            sizes = torch.empty(max(1, len(reqs)) * 2, dtype=torch.int64, device=self.dev)
        outs = {}
        j = 0
        items_init, items_resi = [], []
        for r in inits:
            f = self.fields[r.field]
            st = self._recon(r.client, r.field, s)
            out = self._out_buffer(f)
            outs[r.rid] = out
            items_init.append(dict(**{"in": self._stored_for(f, r.bound)}, out=out, out_size=sizes[j:j + 1],
                                   n_bytes=f.n_bytes, eb1=r.bound, src=st["recon"]))
            st["bound"] = r.bound
            j += 2
        for r in resis:
            f = self.fields[r.field]
            st = self._recon(r.client, r.field, s)
            if st["bound"] is None:
                raise ValueError(f"request {r.rid}: residual before init")
            out = self._out_buffer(f)
            outs[r.rid] = out
            items_resi.append(dict(**{"in": self._stored_for(f, r.bound)}, out=out, out_size=sizes[j:j + 1],
                                   n_bytes=f.n_bytes, eb1=st["bound"], eb2=r.bound, src=st["recon"]))
            st["bound"] = r.bound
            j += 2
        ev0 = torch.cuda.Event(enable_timing=True)
        ev0.record(s)
        with torch.cuda.stream(s):
            if items_init:  # init_send with the client's init_recv fused in
                codec.batch("init_send_apply", items_init, stream=s)
            if items_resi:  # resi_send with the client's resi_recv fused in
                codec.batch("resi_send_apply", items_resi, stream=s)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(s)
        self._timeline.append((ev0, ev))
        return ev, outs, sizes

    # ---------------------------------------------------------------- loops
    def run(self, requests: list[Request], keep_outputs=False):
        """Serves the trace with continuous batching; returns stats."""
        pending = sorted(requests, key=lambda r: r.arrival)
        inflight = []          # (event, reqs, outs, sizes, stream index)
        waiting = []           # arrived, not yet admitted, in arrival order
        busy_clients = set()
        outputs = {}
        self._timeline = []  # (start, end) events of every batch, on its stream
        origin = None
        if self.dev.type == "cuda":
            origin = torch.cuda.Event(enable_timing=True)
            origin.record(self.streams[0])
        t0 = time.perf_counter()
        k = 0
        i = 0
        while i < len(pending) or waiting or inflight:
            now = time.perf_counter() - t0
            # completions
            still = []
            for item in inflight:
                ev, reqs, outs, sizes, _ = item
                if ev.query():
                    tdone = time.perf_counter() - t0
                    for r in reqs:
                        r.done = tdone
                        busy_clients.discard((r.client, r.field))
                    for r in reqs:
                        if keep_outputs:  # handed to the caller, no longer counted
                            outputs[r.rid] = outs[r.rid]
                            self.mem_used -= max_stream_bytes(self.fields[r.field].n_bytes)
                        else:
                            self._free_out.setdefault(r.field, []).append(outs[r.rid])
                else:
                    still.append(item)
            inflight = still
            # admission: in arrival order, except that a request whose client
            # (on that field) has an earlier step running or waiting is passed
            # over, together with that client's later requests
            while i < len(pending) and pending[i].arrival <= now:
                waiting.append(pending[i])
                i += 1
            batch = []
            room = min(self.max_batch, self.max_inflight - sum(len(x[1]) for x in inflight))
            if self.max_batches and len(inflight) >= self.max_batches:
                room = 0
            if room > 0 and waiting:
                held, keep = set(), []
                need_total, claims, new_recons, reloads = 0, {}, set(), set()
                busy_fields = {r.field for x in inflight for r in x[1]}
                for j, r in enumerate(waiting):
                    if len(batch) >= room:
                        keep.extend(waiting[j:])
                        break
                    key = (r.client, r.field)
                    if key in busy_clients or key in held:
                        held.add(key)
                        keep.append(r)
                        continue
                    f = self.fields[r.field]
                    pooled = len(self._free_out.get(r.field, ())) > claims.get(r.field, 0)
                    need = 0 if pooled else max_stream_bytes(f.n_bytes)
                    if f.spilled is not None and r.field not in reloads:
                        need += f.stored_total
                    if not self._resident(key) and key not in new_recons:
                        need += f.n_bytes
                    if self.mem_used + need_total + need > self.mem_cap:
                        protect_f = busy_fields | {b.field for b in batch} | {r.field}
                        protect_c = busy_clients | {key}
                        keep_pool = dict(claims)
                        if pooled:  # the buffer this request will take stays
                            keep_pool[r.field] = keep_pool.get(r.field, 0) + 1
                        if not self._make_room(need_total + need, protect_f, protect_c, keep_pool):
                            keep.extend(waiting[j:])
                            break
                    batch.append(r)
                    busy_clients.add(key)
                    need_total += need
                    if pooled:
                        claims[r.field] = claims.get(r.field, 0) + 1
                    if f.spilled is not None:
                        reloads.add(r.field)
                    if not self._resident(key):
                        new_recons.add(key)
                waiting = keep
            if batch:
                self._tick += 1
                for r in batch:
                    self.fields[r.field].last_use = self._tick
                self._materialize(batch, self.streams[k])
                for r in batch:
                    self.clients[(r.client, r.field)]["last_use"] = self._tick
                ev, outs, sizes = self._launch(k, batch)
                inflight.append((ev, batch, outs, sizes, k))
                k = (k + 1) % len(self.streams)
            elif inflight:
                time.sleep(20e-6)
            elif waiting:  # the head cannot fit even with nothing in flight
                raise RuntimeError(f"request {waiting[0].rid} needs more than the {self.mem_cap}-byte memory cap")
            elif i < len(pending):
                time.sleep(max(0.0, min(1e-3, pending[i].arrival - (time.perf_counter() - t0))))
        for c, s in zip(self.codecs, self.streams):
            c.sync(s)
        wall = time.perf_counter() - t0
        st = self._stats(requests, wall)
        if origin is not None:
            st.update(self._device_timeline(origin, wall))
        return st, outputs

    def _device_timeline(self, origin, wall):
        """Device view of a run from its batches' start and end events: how
        long the GPU had at least one batch running (the union of the batches'
        intervals), as a fraction of the run's wall time, and the median
        batch duration.  Throughput below the device rate with a low busy
        fraction means the host (or another process) left the GPU idle."""
        iv = sorted((origin.elapsed_time(a), origin.elapsed_time(b)) for a, b in self._timeline)
        busy, cur_s, cur_e = 0.0, None, None
        for a, b in iv:
            if cur_e is None or a > cur_e:
                if cur_e is not None:
                    busy += cur_e - cur_s
                cur_s, cur_e = a, b
            else:
                cur_e = max(cur_e, b)
        if cur_e is not None:
            busy += cur_e - cur_s
        dur = sorted(b - a for a, b in iv)
        return {"batches": len(iv), "device_busy_ms": busy,
                "device_busy_frac": busy / (wall * 1e3) if wall > 0 else None,
                "batch_ms_p50": dur[len(dur) // 2] if dur else None}

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
            key = (r.client, r.field)
            need = max_stream_bytes(f.n_bytes) + (f.stored_total if f.spilled else 0) + \
                (0 if self._resident(key) else f.n_bytes)
            if not self._make_room(need, {r.field}, {key}):
                raise RuntimeError(f"request {r.rid} needs more than the {self.mem_cap}-byte memory cap")
            self._tick += 1
            f.last_use = self._tick
            self._materialize([r], s)
            st = self.clients[key]
            st["last_use"] = self._tick
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
                "p99_ms": float(np.percentile(lat, 99) * 1e3) if lat.size else None,
                "spills": self.spills, "reloads": self.reloads}

    def prepare(self, requests: list[Request]):
        """Allocates the reconstruction of every (client, field) the requests
        touch, as a server does when a client opens a field, while they fit
        under the memory cap (the others are allocated at admission), and
        sizes every context's scratch for the largest batch (max_batch
        requests on the largest field), so that serving itself allocates
        only output streams."""
        for r in requests:
            key = (r.client, r.field)
            if not self._resident(key) and self.mem_used + self.fields[r.field].n_bytes <= self.mem_cap:
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
                st["spilled"] = None
            return
        for (c, fname), st in self.clients.items():
            if st["recon"] is not None:
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
