"""Benchmark of the progressive encode/decode path on B200.

Workload: the large-field configuration -- a 512^3 float32 field (512 MiB):
sum of 8 seeded random 3-D sinusoids + N(0, 1e-3^2) noise + 0.1% seeded
outliers at +-1e6 (synthetic; no dataset is named).  One step is one pass of
the whole progressive flow at NOA bounds 1e-2 -> 1e-4 over that field:

    NOA range -> store (1e-4) -> init_send (1e-2) -> init_recv
             -> resi_send (1e-2 -> 1e-4) -> resi_recv

The metric is original-f32 GB/s end to end: field bytes / step time (the
reference's throughput convention, insize * 1e-9 / runtime, applied to the
whole flow; per-operation rates are reported under "ops").  Inputs are larger
than the 126 MB L2, so no flush is needed between steps.

``value`` is timed with CUDA events with the field resident in HBM; the
range stays in device memory and the kernels scale the NOA bounds, so the
steps are enqueued back to back (``value_host_scaled``: the same flow with
the range handed to the host for the scaling, as the reference's drivers
do).  ``e2e``
times the same flow through the C ABI with host buffers: every step copies
the field from pinned host memory to the device and copies the two streams
sent to the client and the final reconstruction back.

--impl reference times the reference path's CPU counterpart (the C oracle,
OpenMP over chunks, all host threads) on the same whole field.  ``ref_cuda``
holds the reference's own CUDA build timed on the same field, bounds and GPU
(its benchmark binaries, inside the clock-sampled window).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "original-f32 GB/s end-to-end at NOA 1e-4, batched/served vs plain; p50/p99 latency"
UNIT = "GB/s"
SHAPE = (512, 512, 512)
EB_STORE, EB_SRC, EB_DST = "1e-4", "1e-2", "1e-4"
# the same field's ABS-mode configuration (finest stored bound, init, residual)
ABS_STORE, ABS_SRC, ABS_DST = "1e-6", "1e-3", "1e-5"
OPS = ("noa_range", "store", "init_send", "init_recv", "resi_send", "resi_recv")
FIVE = OPS[1:]  # the encode/decode operations (the reference's binaries time these)
# the step with each send fused with the client's receive
FUSED_OPS = ("noa_range", "store", "init_send_apply", "resi_send_apply")


def make_field(seed: int, device, shape=SHAPE, outliers: bool = True) -> torch.Tensor:
    from cortado_b200 import fields
    return fields.sinusoid(shape, seed, outlier_frac=1e-3 if outliers else 0.0, device=device).reshape(-1)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------- GPU arm
class Flow:
    """Preallocated buffers and the six calls of one step on one stream.

    device_noa: the range stays in device memory and the NOA entry points
    scale the bounds in the kernels, so nothing in a step waits for the host
    (the same streams as the host-scaled calls); False: the range is handed
    to the host, which scales the bounds, as the reference's drivers do."""

    def __init__(self, codec, x: torch.Tensor, stream: torch.cuda.Stream, abs_mode: bool = False,
                 device_noa: bool = True, fused: bool = False):
        from cortado_b200 import ops
        self.c, self.x, self.s, self.abs_mode = codec, x, stream, abs_mode
        self.device_noa = device_noa
        self.fused = fused  # NOA, device bounds: sends fused with the receives (the client's floats in fin)
        self.ops = FUSED_OPS if fused else OPS
        self.mm = torch.empty(2, dtype=torch.float32, device=x.device)
        self.stream = stream  # the compute stream, as cortado_b200.pipeline expects
        dev = x.device
        self.n = x.numel() * 4
        cap = ops.max_stream_bytes(self.n)
        self.stor = torch.empty(cap, dtype=torch.uint8, device=dev)
        self.init = torch.empty(cap, dtype=torch.uint8, device=dev)
        self.resi = torch.empty(cap, dtype=torch.uint8, device=dev)
        self.cl = torch.empty_like(x)
        self.fin = torch.empty_like(x)
        self.sizes = torch.zeros(8, dtype=torch.int64, device=dev)
        self.ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(self.ops) + 1)]

    def bounds(self):
        from cortado_b200 import storage
        lo, hi = self.c.INOA_find_range(self.x, stream=self.s)  # run in both modes, as the reference's store does
        if self.abs_mode:
            return tuple(float(storage.f32(e)) for e in (ABS_STORE, ABS_SRC, ABS_DST))
        rng = storage.value_range(lo, hi)
        return (float(storage.noa_scale(EB_STORE, rng)), float(storage.noa_scale(EB_SRC, rng)),
                float(storage.noa_scale(EB_DST, rng)))

    def step(self, timed=False):
        if self.device_noa:
            return self.step_device_noa(timed)
        c, s, sz = self.c, self.s, self.sizes
        if timed:
            self.ev[0].record(s)
        eb_store, eb_src, eb_dst = self.bounds()  # NOA range (synchronous min/max)
        if timed:
            self.ev[1].record(s)
        c.server_encode(self.x, self.n, self.stor, sz[0:1], eb_store, stream=s)
        if timed:
            self.ev[2].record(s)
        c.s2c_encode(self.stor, self.init, sz[1:2], eb_src, self.n, stream=s)
        if timed:
            self.ev[3].record(s)
        c.client_decode(self.init, self.cl, sz[2:3], stream=s)
        if timed:
            self.ev[4].record(s)
        c.residual_encode(self.stor, self.resi, sz[3:4], eb_src, eb_dst, self.n, stream=s)
        if timed:
            self.ev[5].record(s)
        c.residual_apply(self.cl, self.n, self.resi, self.fin, sz[4:5], stream=s)
        if timed:
            self.ev[6].record(s)

    def step_device_noa(self, timed=False):
        from cortado_b200 import storage
        c, s, sz, mm = self.c, self.s, self.sizes, self.mm
        ev = self.ev if timed else [None] * len(self.ev)
        rec = (lambda i: ev[i].record(s)) if timed else (lambda i: None)
        rec(0)
        c.INOA_find_range_device(self.x, mm, stream=s)  # computed in both modes, as the reference's store does
        rec(1)
        if self.fused:
            a, b, d = (float(storage.f32(e)) for e in (EB_STORE, EB_SRC, EB_DST))
            c.server_encode_noa(self.x, self.n, self.stor, sz[0:1], mm, a, stream=s)
            rec(2)
            c.s2c_encode_apply_noa(self.stor, self.init, sz[1:2], mm, b, self.n, self.fin, stream=s)
            rec(3)
            c.residual_encode_apply_noa(self.stor, self.resi, sz[3:4], mm, b, d, self.n, self.fin, stream=s)
            rec(4)
            return
        if self.abs_mode:
            a, b, d = (float(storage.f32(e)) for e in (ABS_STORE, ABS_SRC, ABS_DST))
            c.server_encode(self.x, self.n, self.stor, sz[0:1], a, stream=s)
            rec(2)
            c.s2c_encode(self.stor, self.init, sz[1:2], b, self.n, stream=s)
            rec(3)
            c.client_decode(self.init, self.cl, sz[2:3], stream=s)
            rec(4)
            c.residual_encode(self.stor, self.resi, sz[3:4], b, d, self.n, stream=s)
        else:
            a, b, d = (float(storage.f32(e)) for e in (EB_STORE, EB_SRC, EB_DST))
            c.server_encode_noa(self.x, self.n, self.stor, sz[0:1], mm, a, stream=s)
            rec(2)
            c.s2c_encode_noa(self.stor, self.init, sz[1:2], mm, b, self.n, stream=s)
            rec(3)
            c.client_decode(self.init, self.cl, sz[2:3], stream=s)
            rec(4)
            c.residual_encode_noa(self.stor, self.resi, sz[3:4], mm, b, d, self.n, stream=s)
        rec(5)
        c.residual_apply(self.cl, self.n, self.resi, self.fin, sz[4:5], stream=s)
        rec(6)

    def op_ms(self):
        return [self.ev[i].elapsed_time(self.ev[i + 1]) for i in range(len(self.ops))]


def run_gpu(args, rank, world):
    # clocks are sampled from before the warm-up until after the last timed
    # region (the main, end-to-end and ABS timings all fall inside)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
        r = _run_gpu(args, rank, world)
    r["clocks"] = dict(clk.summary(), window="warm-up through the last timed region")
    return r


def _run_gpu(args, rank, world):
    import tempfile
    from cortado_b200 import autotune, ops
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    x = make_field(2 + rank, dev, args.shape)
    # The autotuner picks every operation's launch parameters on this GPU for
    # the workload's size class (untimed, before the warm-up), into a cache
    # private to this run that every later context of the process applies.
    os.environ["CORTADO_TUNE_CACHE"] = os.path.join(tempfile.mkdtemp(prefix="cortado_tune_"), "tune.json")
    codec = ops.Codec(dev.index)
    tuning = autotune.tune(codec, n_bytes=x.numel() * 4) if not args.no_tune else None
    if tuning is not None:
        autotune.save_cache({autotune.key(dev, x.numel() * 4): tuning})
    stream = torch.cuda.Stream(dev)
    fl = Flow(codec, x, stream)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            fl.step()
        codec.sync(stream)
        # correctness guard on the timed configuration: the final
        # reconstruction must equal iCQ(CQ(x)) at the destination bound
        _, _, eb_dst = fl.bounds()
        ok = bool(torch.all((fl.fin - x).abs() <= eb_dst))
        sizes = fl.sizes.cpu().tolist()
    barrier(world)
    torch.cuda.synchronize(dev)
    def timed_steps(flow, k):
        """k steps enqueued back to back (the device-NOA flow waits for nothing
        on the host), each with its own events; returns (ms per step, mean ms
        per operation)."""
        sets = [[torch.cuda.Event(enable_timing=True) for _ in range(len(flow.ops) + 1)] for _ in range(k)]
        st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(flow.s):
            st.record(flow.s)
            for evs in sets:
                flow.ev = evs
                flow.step(timed=True)
            en.record(flow.s)
            torch.cuda.synchronize(dev)
        ops = np.mean([[e[i].elapsed_time(e[i + 1]) for i in range(len(flow.ops))] for e in sets], axis=0)
        return st.elapsed_time(en) / k, ops

    ms, per_op = timed_steps(fl, args.steps)
    codec.sync(stream)
    ms = max_over_ranks(ms, world, dev)
    n = fl.n
    # the same flow with the range handed to the host, which scales the bounds
    # (the reference drivers' way; every step waits for the device once)
    fh = Flow(codec, x, stream, device_noa=False)
    with torch.cuda.stream(stream):
        fh.step()
        codec.sync(stream)
    ms_host, per_op_host = timed_steps(fh, args.steps)
    codec.sync(stream)
    ms_host = max_over_ranks(ms_host, world, dev)
    del fh
    # the same step with each send fused with the client's receive (a server
    # that keeps the client's reconstruction on this GPU): four launches, the
    # same streams and the same final reconstruction
    ff = Flow(codec, x, stream, fused=True)
    with torch.cuda.stream(stream):
        ff.step()
        codec.sync(stream)
    s_i, s_r = int(fl.sizes[1]), int(fl.sizes[3])
    fused_ok = (int(ff.sizes[1]) == s_i and int(ff.sizes[3]) == s_r and torch.equal(ff.init[:s_i], fl.init[:s_i])
                and torch.equal(ff.resi[:s_r], fl.resi[:s_r])
                and torch.equal(ff.fin.view(torch.int32), fl.fin.view(torch.int32)))
    ms_fused, per_op_fused = timed_steps(ff, args.steps)
    codec.sync(stream)
    ms_fused = max_over_ranks(ms_fused, world, dev)
    del ff

    # Reference-style timing of each operation: the host clock around one call
    # and a stream synchronize, median of 10 after a warm-up, as the
    # reference's benchmark binaries time their wrappers.  Each call repeats
    # an operation of the step above on the same inputs.
    eb_store, eb_src, eb_dst = fl.bounds()
    c_, s_, sz_ = fl.c, fl.s, fl.sizes
    ref_calls = {
        "noa_range": lambda: fl.bounds(),
        "store": lambda: c_.server_encode(fl.x, n, fl.stor, sz_[0:1], eb_store, stream=s_),
        "init_send": lambda: c_.s2c_encode(fl.stor, fl.init, sz_[1:2], eb_src, n, stream=s_),
        "init_recv": lambda: c_.client_decode(fl.init, fl.cl, sz_[2:3], stream=s_),
        "resi_send": lambda: c_.residual_encode(fl.stor, fl.resi, sz_[3:4], eb_src, eb_dst, n, stream=s_),
        "resi_recv": lambda: c_.residual_apply(fl.cl, n, fl.resi, fl.fin, sz_[4:5], stream=s_),
    }
    ref_style = {}
    with torch.cuda.stream(stream):
        for name, fn in ref_calls.items():
            fn()
            stream.synchronize()
            ts = []
            for _ in range(10):
                t0 = time.perf_counter()
                fn()
                stream.synchronize()
                ts.append((time.perf_counter() - t0) * 1e3)
            ref_style[name] = float(np.median(ts))
    codec.sync(stream)

    # e2e through the C ABI with host buffers: every step copies the field in
    # from pinned host memory and both streams and the final reconstruction
    # back, scheduled by cortado_b200.pipeline: two flows (own buffers,
    # context and compute stream) alternate, copies in run one step ahead on
    # their own stream and copies out on another, so a step's copies out
    # overlap the next step's copy in and compute.
    from cortado_b200.pipeline import Pipeline
    hx = x.cpu().pin_memory()
    s_init, s_resi = int(sizes[1]), int(sizes[3])
    codec2 = ops.Codec(dev.index)
    stream2 = torch.cuda.Stream(dev)
    flows = [Flow(codec, fl.x, stream), Flow(codec2, torch.empty_like(x), stream2)]
    hbufs = [(torch.empty(s_init, dtype=torch.uint8).pin_memory(), torch.empty(s_resi, dtype=torch.uint8).pin_memory(),
              torch.empty(x.numel(), dtype=torch.float32).pin_memory()) for _ in flows]

    def load(i, f, s):
        f.x.copy_(hx, non_blocking=True)

    def run(i, f, s):
        f.step()

    def store(i, f, s):
        h_init, h_resi, h_fin = hbufs[i % 2]
        h_init.copy_(f.init[:s_init], non_blocking=True)
        h_resi.copy_(f.resi[:s_resi], non_blocking=True)
        h_fin.copy_(f.fin, non_blocking=True)

    pipe = Pipeline(dev, flows, load, run, store)
    e_steps = max(2, min(args.steps, 6))
    pipe(2)
    pipe.sync()
    barrier(world)
    torch.cuda.synchronize(dev)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(pipe.s_in)
    pipe(e_steps)
    end.record(pipe.s_out)
    torch.cuda.synchronize(dev)
    e2e_ok = bool(torch.equal(hbufs[0][2], fl.fin.cpu())) and bool(torch.equal(hbufs[1][2], hbufs[0][2]))
    e2e_ms = max_over_ranks(start.elapsed_time(end) / e_steps, world, dev)
    # The same schedule with no device work between the copies: the time of
    # the copies alone, the PCIe floor of the end-to-end step.
    pipe0 = Pipeline(dev, flows, load, lambda i, f, s: None, store)
    pipe0(2)
    pipe0.sync()
    barrier(world)
    torch.cuda.synchronize(dev)
    start.record(pipe0.s_in)
    pipe0(e_steps)
    end.record(pipe0.s_out)
    torch.cuda.synchronize(dev)
    copy_ms = max_over_ranks(start.elapsed_time(end) / e_steps, world, dev)
    codec.sync(stream)
    codec2.sync(stream2)
    codec2.close()
    ok = ok and e2e_ok

    # ABS-mode pass over the same field (secondary report)
    fa = Flow(codec, x, stream, abs_mode=True)
    with torch.cuda.stream(stream):
        for _ in range(2):
            fa.step()
        codec.sync(stream)
        _, _, eb_a = fa.bounds()
        abs_ok = bool(torch.all((fa.fin - x).abs() <= eb_a))
        abs_sizes = fa.sizes.cpu().tolist()
        a_steps = max(1, min(args.steps, 5))
        barrier(world)
        torch.cuda.synchronize(dev)
    abs_ms, a_op = timed_steps(fa, a_steps)
    abs_ms = max_over_ranks(abs_ms, world, dev)
    codec.sync(stream)
    abs_res = dict(ms=abs_ms, per_op=a_op, sizes=abs_sizes, ok=abs_ok)
    del fa

    # The NOA flow on the same generator without the outliers (sinusoids and
    # noise only, as in the small-field configuration) at this shape: the NOA
    # range is the signal's own, so the streams are dense.
    xd = make_field(2 + rank, dev, args.shape, outliers=False)
    torch.cuda.synchronize(dev)  # generated on the default stream; the flow runs on its own
    fd = Flow(codec, xd, stream)
    with torch.cuda.stream(stream):
        for _ in range(2):
            fd.step()
        codec.sync(stream)
        _, _, eb_d = fd.bounds()
        dense_ok = bool(torch.all((fd.fin - xd).abs() <= eb_d))
        dense_sizes = fd.sizes.cpu().tolist()
        barrier(world)
        torch.cuda.synchronize(dev)
    dense_ms, d_op = timed_steps(fd, a_steps)
    dense_ms = max_over_ranks(dense_ms, world, dev)
    codec.sync(stream)
    dense_res = dict(ms=dense_ms, per_op=d_op, sizes=dense_sizes, ok=dense_ok)
    del fd, xd
    x_host = x.cpu().numpy()
    # The reference's own CUDA build on the same field, bounds and GPU, in the
    # same clock-sampled window (a reported baseline; one GPU only).
    ref_cuda = None
    if world == 1 and not args.no_ref_cuda:
        ref_cuda = reference_cuda_baseline(x_host)
    return dict(abs=abs_res, dense=dense_res, sms=torch.cuda.get_device_properties(dev).multi_processor_count,
                ms=ms, per_op=per_op, n=n, sizes=sizes, ok=ok, e2e_ms=e2e_ms, copy_ms=copy_ms, ref_style=ref_style,
                ms_host=ms_host, per_op_host=per_op_host, ms_fused=ms_fused, per_op_fused=per_op_fused,
                fused_ok=fused_ok,
                h2d=n, d2h=s_init + s_resi + n, x_host=x_host, ref_cuda=ref_cuda, tuning=tuning)


def barrier(world):
    if world > 1:
        torch.distributed.barrier()


def max_over_ranks(v, world, dev):
    """Slowest rank's time (every rank takes part; device = the rank's device,
    or cpu under gloo)."""
    if world == 1:
        return v
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_gbs(field_bytes: int, world: int, ms_per_step: float) -> float:
    """Whole-job original-data rate: every rank processes its own field."""
    return world * field_bytes * 1e-9 / (ms_per_step * 1e-3)


def bench_batched(codec, dev, n_fields=64, seed=3, max_mb=256, bounds=("1e-1", "1e-2", "1e-3", "1e-4")):
    """Many-fields configuration: n_fields float32 fields of log-uniform size
    1 MiB .. max_mb MiB (multiples of 4 B, mixed generators), each stored at 4
    NOA bounds -- one batched launch vs one launch per (field, bound)."""
    from cortado_b200 import fields, storage
    from cortado_b200.ops import max_stream_bytes
    xs = [fields.mixed_field(nf, kind, fs, device=dev)
          for nf, kind, fs in fields.field_set(n_fields, seed, 1 << 20, max_mb << 20)]
    items, outs = [], []
    sizes = torch.zeros(len(xs) * len(bounds), dtype=torch.int64, device=dev)
    for i, x in enumerate(xs):
        lo, hi = codec.INOA_find_range(x)
        r = storage.value_range(lo, hi)
        for j, b in enumerate(bounds):
            k = i * len(bounds) + j
            out = torch.empty(max_stream_bytes(x.numel() * 4), dtype=torch.uint8, device=dev)
            outs.append(out)
            items.append(dict(**{"in": x}, out=out, out_size=sizes[k:k + 1], n_bytes=x.numel() * 4,
                              eb1=float(storage.noa_scale(b, r))))
    total = sum(it["n_bytes"] for it in items)

    def plain():
        for it in items:
            codec.server_encode(it["in"], it["n_bytes"], it["out"], it["out_size"], it["eb1"])

    def batched():
        codec.batch("store", items)

    res = {}
    for name, fn in (("plain", plain), ("batched", batched)):
        fn()
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ts = []
        for _ in range(3):
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize(dev)
            ts.append(s.elapsed_time(e))
        res[name] = {"ms": float(np.median(ts)), "orig_GBps": total * 1e-9 / (np.median(ts) * 1e-3)}
    codec.sync()
    del outs
    return {"workload": f"{n_fields} fields 1-{max_mb} MiB log-uniform (mixed sinusoid/GRF k^-3/white), "
                        f"stored at NOA {list(bounds)}: {len(items)} encodes", "field_bytes_total": total // len(bounds),
            **res, "speedup": res["plain"]["ms"] / res["batched"]["ms"]}


def bench_serving(dev, n_fields=32, n_requests=400, rates=(2000.0, 8000.0, 32000.0, None), seed=5, max_mb=512):
    """Serving configuration: resident stored fields (4..max_mb MiB, mixed
    generators), Poisson arrivals (60% init at NOA 1e-1..1e-3, 40% residual 1-3
    decades finer); continuous batching vs the plain per-request pipeline at a
    swept arrival rate.  The same request sequence is replayed at every rate
    (arrival times scaled), three times per rate; rate None queues every
    request at the start, so the aggregate GB/s there is each pipeline's
    capacity."""
    from cortado_b200 import fields, storage
    from cortado_b200.serve import Server, poisson_trace
    rng = np.random.Generator(np.random.PCG64(seed))
    srv = Server(dev.index, mem_cap_bytes=120 * 10**9, max_inflight=64, n_streams=3, max_batch=16)
    ranges = {}
    for i, (nf, kind, fs) in enumerate(fields.field_set(n_fields, seed, 4 << 20, max_mb << 20, rng=rng)):
        x = fields.mixed_field(nf, kind, fs, device=dev)
        r = float(x.max() - x.min())
        ranges[f"f{i}"] = r
        srv.add_field(f"f{i}", x, [float(storage.noa_scale(e, r)) for e in (1e-1, 1e-3, 1e-5, 1e-7)])
    trace = poisson_trace(rng, srv.fields, n_requests, 1.0, n_clients=16, ranges=ranges)
    unit_arrivals = [r.arrival for r in trace]  # at one request per second
    # Client reconstructions are allocated up front (a server does that when a
    # client opens a field); each mode serves the trace once untimed at the
    # backlog point (the most requests in flight), so the allocator holds its
    # output streams, then once measured per rate, from fresh client progress
    # on the same buffers.
    srv.prepare(trace)

    def once(fn, rate):
        srv.reset_clients(free=False)
        for r, u in zip(trace, unit_arrivals):
            r.done = -1.0
            r.arrival = u / rate if rate else 0.0
        a0 = torch.cuda.memory_stats(dev).get("num_device_alloc", 0)
        st = fn(trace)[0]
        st["device_allocs"] = torch.cuda.memory_stats(dev).get("num_device_alloc", 0) - a0
        return st

    once(srv.run, None)
    once(srv.run_plain, None)
    # Every rate three times, served and plain; each entry is the run with
    # the median ratio, and `ratios` lists all three (a run that the host
    # stalled shows there, with a low device busy fraction).
    sweep = []
    for rate in rates:
        runs = [(once(srv.run, rate), once(srv.run_plain, rate)) for _ in range(3)]
        runs.sort(key=lambda sp: sp[0]["orig_GBps"] / sp[1]["orig_GBps"])
        served, plain = runs[1]
        sweep.append({"rate_hz": rate if rate else "backlog", "served": served, "plain": plain,
                      "speedup": served["orig_GBps"] / plain["orig_GBps"],
                      "ratios": [sp[0]["orig_GBps"] / sp[1]["orig_GBps"] for sp in runs]})
    srv.close()
    cap = sweep[-1]  # the capacity point (every request queued at the start)
    return {"workload": f"{n_fields} resident fields 4-{max_mb} MiB, {n_requests} requests, Poisson arrivals at "
                        f"{[s['rate_hz'] for s in sweep]} per s, 60% init / 40% residual",
            "sweep": sweep, "served": cap["served"], "plain": cap["plain"], "speedup": cap["speedup"],
            "capacity_ratios": cap["ratios"]}


def bench_chain(codec, dev, side=16384, seed=4, reps=5):
    """Progressive-chain configuration: a side x side float32 Gaussian random
    field with spectrum k^-2.5 (1 GiB at 16384^2), stored at NOA 1e-1, 1e-3,
    1e-5, 1e-7; a client's init at 1e-1, then residual steps to 1e-2 ... 1e-6,
    each applied and bound-checked on the device, the whole sequence captured
    as one CUDA graph.  Original-data GB/s counts the field once per step."""
    from cortado_b200 import fields, storage
    from cortado_b200.chain import ProgressiveChain
    x = fields.grf((side, side), seed, slope=2.5, device=dev).reshape(-1)
    lo, hi = codec.INOA_find_range(x)
    rng = storage.value_range(lo, hi)
    nb = lambda e: float(storage.noa_scale(e, rng))  # noqa: E731
    ch = ProgressiveChain(codec, x, [nb(e) for e in (1e-1, 1e-3, 1e-5, 1e-7)], nb(1e-1),
                          [nb(e) for e in (1e-2, 1e-3, 1e-4, 1e-5, 1e-6)])
    ch.capture()  # runs the chain eagerly once first

    def timed(fn):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fn()
        torch.cuda.synchronize(dev)
        ts = []
        for _ in range(reps):
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize(dev)
            ts.append(s.elapsed_time(e))
        return float(np.median(ts))

    eager_ms = timed(ch.run_eager)
    graph_ms = timed(ch.replay)
    codec.sync()
    ok = bool((ch.first_bad == -1).all().item())
    n, steps = ch.n, len(ch.bounds)
    res = {"workload": f"{side}x{side} float32 GRF k^-2.5 ({n >> 20} MiB), stored at NOA 1e-1/1e-3/1e-5/1e-7; "
                       "init 1e-1, residual steps to 1e-2 ... 1e-6, each applied and bound-checked on the device",
           "steps": steps, "launches": ch.launches(), "graph_ms": graph_ms, "eager_ms": eager_ms,
           "orig_GBps": n * steps * 1e-9 / (graph_ms * 1e-3), "bounds_verified": ok,
           "stream_bytes": [int(v) for v in ch.stream_sizes.tolist()]}
    del ch, x
    return res


def load_profile(name):
    p = os.path.join(ROOT, "profiles", name)
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def load_traffic():
    return load_profile("traffic.json")


def kernel_fracs(n, sizes, per_op, peak):
    """Algorithmic HBM bytes of each kernel's launch (its input read once,
    its output written once), its duration, and their rate as a fraction of
    the copy peak."""
    s_stor, s_init, s_resi = sizes[0], sizes[1], sizes[3]
    alg = {"store": n + s_stor, "init_send": s_stor + s_init, "init_recv": s_init + n,
           "resi_send": s_stor + s_resi, "resi_recv": 2 * n + s_resi, "noa_range": n}
    op_ms = dict(zip(OPS, [float(v) for v in per_op]))
    return alg, op_ms, {k: alg[k] / (op_ms[k] * 1e-3) * 1e-9 / peak for k in alg}


def issue_fracs(n, op_ms, sms, sm_mhz):
    """The re-encoders move only compressed bytes, so their bound is the
    instruction issue rate: warp instructions per chunk (from the ncu capture
    of the NOA flow in profiles/issue.json) x chunks, over 4 issues per SM per
    cycle at the sampled median SM clock, divided by the measured time."""
    ipc = load_profile("issue.json").get("inst_per_chunk", {})
    if not sm_mhz:
        return None
    chunks = (n + 16383) // 16384
    return {k: ipc[k] * chunks / (sms * 4 * sm_mhz * 1e6) / (op_ms[k] * 1e-3)
            for k in ("init_send", "resi_send") if k in ipc}


def host_field(shape, seed=2, sample_mb=0) -> np.ndarray:
    """The benchmark field's bytes in host memory, generated on the GPU when
    one is present (the same bytes the GPU arm times), else on the CPU.
    sample_mb > 0 builds a smaller field of about that many MiB instead (the
    same generator on fewer z-planes; CPU tests only)."""
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    if sample_mb > 0:
        shape = (max(1, sample_mb * (1 << 20) // (4 * shape[1] * shape[2])), shape[1], shape[2])
    return make_field(seed, dev, shape).cpu().numpy()


def cpu_step(x: np.ndarray, threads: int) -> float:
    """One step of the benchmark flow (NOA range, store, init_send, init_recv,
    resi_send, resi_recv) through the CPU oracle on `threads` host threads;
    returns its duration in seconds."""
    from cortado_b200 import storage
    from oracle import oracle as O
    t0 = time.perf_counter()
    rng = O.noa_range(x)
    eb_s, eb_a, eb_b = (float(storage.noa_scale(e, rng)) for e in (EB_STORE, EB_SRC, EB_DST))
    stor = O.store_encode(x, eb_s, threads)
    init = O.init_send(stor, eb_a, threads)
    cl = O.init_recv(init, threads)
    resi = O.resi_send(stor, eb_a, eb_b, threads)
    O.resi_recv(cl, resi, threads)
    return time.perf_counter() - t0


def cpu_baseline(x: np.ndarray, steps=1, warmup=1, threads=None):
    """The C oracle (OpenMP over chunks, all host threads) on the whole
    benchmark field: `warmup` untimed steps, then `steps` timed ones."""
    threads = threads or os.cpu_count()
    for _ in range(warmup):
        cpu_step(x, threads)
    total = sum(cpu_step(x, threads) for _ in range(steps))
    ms = total * 1e3 / steps
    return {"value": x.nbytes * 1e-9 / (ms * 1e-3), "unit": UNIT, "cores": threads, "kind": "port",
            "ms_per_step": ms, "steps": steps,
            "sample": f"the whole field ({x.nbytes} bytes), every operation of the step, {steps} timed step(s) "
                      f"after {warmup} warm-up"}


def reference_cuda_baseline(x: np.ndarray, timeout_s=120):
    """The reference's own CUDA build (its benchmark binaries, compiled from its
    sources for sm_100a into oracle/_ref) on the same field and bounds, NOA
    and ABS: each operation's median of 10 runs as those binaries report it
    (host-side timer around the wrapper, which allocates and frees its carry
    array per call; src/cortado_store.cu:239-245, src/cortado_init.cu:448,549,
    src/cortado_resi.cu:509,641).  A reported baseline, never the measured
    product."""
    import re
    import shutil
    import tempfile
    ref = os.path.join(ROOT, "oracle", "_ref")
    bins = {b: os.path.join(ref, b) for b in ("store_bench", "init_bench", "resi_bench")}
    if not all(os.access(p, os.X_OK) for p in bins.values()):
        return {"unavailable": "oracle/_ref benchmark binaries not built (the reference sources were absent at build)"}
    d = tempfile.mkdtemp(prefix="cortado_refcuda_")
    f = os.path.join(d, "field.f32")
    x.tofile(f)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s)
        if r.returncode != 0:
            raise RuntimeError(f"{os.path.basename(cmd[0])} rc={r.returncode}: {r.stderr[-300:]}")
        return r.stdout

    def msecs(out, key):
        m = re.findall(rf"^{key}:\s+([0-9.]+) s", out, re.M)
        return float(m[-1]) * 1e3 if m else None

    res = {"kind": "reference CUDA build", "runs": 10,
           "timer": "the reference binaries' own: median of 10 runs after a warm-up, wrapper-inclusive"}
    try:
        for mode, (st, a, b), flag in (("noa", (EB_STORE, EB_SRC, EB_DST), []),
                                       ("abs", (ABS_STORE, ABS_SRC, ABS_DST), ["-a"])):
            o1 = run([bins["store_bench"], f, st, "-r", "10", *flag])
            o2 = run([bins["init_bench"], f, st, a, "-r", "10", *flag])
            o3 = run([bins["resi_bench"], f, st, a, b, "-r", "10", *flag])
            ops = {"store": msecs(o1, "runtime"), "init_send": msecs(o2, "send runtime"),
                   "init_recv": msecs(o2, "recv runtime"), "resi_send": msecs(o3, "send runtime"),
                   "resi_recv": msecs(o3, "recv runtime")}
            if any(v is None for v in ops.values()):
                raise RuntimeError(f"no runtime line in the {mode} output")
            res[mode] = {"ms": ops, "sum_ms": sum(ops.values())}
    except (RuntimeError, subprocess.TimeoutExpired, OSError) as e:
        res = {"unavailable": f"reference binaries failed: {e}"}
    finally:
        shutil.rmtree(d, ignore_errors=True)
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cortado_b200", choices=["cortado_b200", "reference"])
    ap.add_argument("--cpu-sample-mb", type=int, default=0,
                    help="CPU legs on a smaller field of about this many MiB (0: the whole field)")
    ap.add_argument("--no-ref-cuda", action="store_true", help="skip timing the reference's CUDA build")
    ap.add_argument("--no-tune", action="store_true", help="keep the shipped launch parameters (no tuning run)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shape", default="512,512,512", help="field shape (profiling uses a smaller one)")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched, serving and chain measurements")
    ap.add_argument("--extras", default="batched,serving,chain", help="which of those to run (comma list)")
    ap.add_argument("--batched-fields", type=int, default=64, help="fields of the batched measurement")
    ap.add_argument("--batched-max-mb", type=int, default=256, help="largest field of the batched measurement")
    args = ap.parse_args()
    extras = set() if args.no_extras else {e for e in args.extras.split(",") if e}
    args.shape = tuple(int(v) for v in args.shape.split(","))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    cfg = {"workload": "512^3 float32 field (512 MiB), 8 random sinusoids + N(0,1e-3) noise + 0.1% +-1e6 outliers; "
                       "step = NOA range, store 1e-4, init_send 1e-2, init_recv, resi_send 1e-2->1e-4, resi_recv",
           "field_bytes": int(np.prod(args.shape)) * 4, "shape": list(args.shape), "bounds_noa": {"store": EB_STORE, "init": EB_SRC, "resi": [EB_SRC, EB_DST]},
           "parallelism": f"replicas{args.gpus} (independent fields, no collective)",
           "l2": "inputs larger than L2 (no flush needed)"}

    if args.impl == "reference":
        if rank != 0:
            return
        x = host_field(args.shape, 2, args.cpu_sample_mb)
        k = max(1, args.steps)
        base = cpu_baseline(x, steps=k, warmup=args.warmup)
        v = base["value"]
        cfg["field_bytes"] = int(x.nbytes)
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
                          "steps": k, "warmup": args.warmup, "ms_per_step": base["ms_per_step"],
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32/f32",
                          "data": "synthetic", "config": cfg, "cpu_baseline": base,
                          "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    r = run_gpu(args, rank, world)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    n = r["n"]
    gbs = job_gbs(n, world, r["ms"])
    ops_gbs = {op: (n * 1e-9 / (t * 1e-3) if t > 0 else None) for op, t in zip(OPS, r["per_op"])}
    sizes = r["sizes"]
    s_stor, s_init, s_resi = sizes[0], sizes[1], sizes[3]
    peak, peak_kind = peaks()
    alg, op_ms, fracs = kernel_fracs(n, sizes, r["per_op"], peak)
    _, abs_ms, abs_fracs = kernel_fracs(n, r["abs"]["sizes"], r["abs"]["per_op"], peak)
    _, dense_ms, dense_fracs = kernel_fracs(n, r["dense"]["sizes"], r["dense"]["per_op"], peak)
    dom = max(alg, key=lambda k: op_ms[k])
    achieved = alg[dom] / (op_ms[dom] * 1e-3) * 1e-9
    traffic = load_traffic().get(dom)
    line = {
        "metric": METRIC, "value": gbs, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32/f32", "data": "synthetic", "config": cfg,
        "ops": {k: {"ms": op_ms[k], "orig_GBps": ops_gbs[k]} for k in OPS},
        # host clock around call + synchronize, median of 10 (the reference binaries' convention)
        "ops_reference_style_ms": r["ref_style"],
        "stream_bytes": {"stor": s_stor, "init": s_init, "resi": s_resi},
        "bounds_verified": r["ok"],
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "per_kernel_frac": fracs,
                     "per_kernel_frac_abs": abs_fracs,
                     "per_kernel_frac_no_outliers": dense_fracs,
                     # the re-encoders' own bound: the fraction of the SMs' issue rate
                     "issue_frac": issue_fracs(n, op_ms, r["sms"], r["clocks"].get("sm_mhz"))},
        "fused_flow": {"what": "the same step with init_send and resi_send each fused with the client's receive "
                               "(the client's reconstruction kept on this GPU): range, store, init_send_apply, "
                               "resi_send_apply",
                       "value": job_gbs(n, world, r["ms_fused"]), "ms_per_step": r["ms_fused"],
                       "ops_ms": dict(zip(FUSED_OPS, [float(v) for v in r["per_op_fused"]])),
                       # algorithmic bytes: the stored stream in, the stream out, the
                       # client's floats written (init) or read and written (resi)
                       "per_kernel_frac": {
                           "init_send_apply": (s_stor + s_init + n) / (r["per_op_fused"][2] * 1e-3) * 1e-9 / peak,
                           "resi_send_apply": (s_stor + s_resi + 2 * n) / (r["per_op_fused"][3] * 1e-3) * 1e-9 / peak},
                       "matches_plain": r["fused_ok"]},
        # the same flow with the range handed to the host for the bounds' scaling
        "value_host_scaled": {"value": job_gbs(n, world, r["ms_host"]), "ms_per_step": r["ms_host"],
                              "ops_ms": dict(zip(OPS, [float(v) for v in r["per_op_host"]]))},
        "e2e": {"value": world * n * 1e-9 / (r["e2e_ms"] * 1e-3), "unit": UNIT, "h2d_bytes_per_step": r["h2d"],
                "d2h_bytes_per_step": r["d2h"], "ms_per_step": r["e2e_ms"],
                # the same copies on the same schedule without the device work
                "copy_floor": {"ms_per_step": r["copy_ms"], "value": world * n * 1e-9 / (r["copy_ms"] * 1e-3),
                               "h2d_GBps": r["h2d"] * 1e-9 / (r["copy_ms"] * 1e-3),
                               "d2h_GBps": r["d2h"] * 1e-9 / (r["copy_ms"] * 1e-3)},
                "frac_of_copy_floor": r["copy_ms"] / r["e2e_ms"]},
        # one kernel per operation, two for the NOA range (min/max, hand-over)
        "gpu_launches": args.steps * (len(OPS) + 1),
        "abs_mode": {"bounds_abs": {"store": ABS_STORE, "init": ABS_SRC, "resi": [ABS_SRC, ABS_DST]},
                     "value": job_gbs(n, world, r["abs"]["ms"]), "ms_per_step": r["abs"]["ms"],
                     "bounds_verified": r["abs"]["ok"],
                     "stream_bytes": {"stor": r["abs"]["sizes"][0], "init": r["abs"]["sizes"][1],
                                      "resi": r["abs"]["sizes"][3]},
                     "ops": {k: {"ms": t, "orig_GBps": n * 1e-9 / (t * 1e-3) if t > 0 else None}
                             for k, t in abs_ms.items()}},
        "no_outliers": {"workload": "the same generator without the outliers (8 sinusoids + N(0,1e-3) noise) at the "
                                    "same shape, NOA bounds as above",
                        "value": job_gbs(n, world, r["dense"]["ms"]), "ms_per_step": r["dense"]["ms"],
                        "bounds_verified": r["dense"]["ok"],
                        "stream_bytes": {"stor": r["dense"]["sizes"][0], "init": r["dense"]["sizes"][1],
                                         "resi": r["dense"]["sizes"][3]},
                        "ops": {k: {"ms": t, "orig_GBps": n * 1e-9 / (t * 1e-3) if t > 0 else None}
                                for k, t in dense_ms.items()}},
        "clocks": r["clocks"],
    }
    if r["tuning"] is not None:
        line["tuning"] = {"source": "tuned on this GPU for the workload's size class before the warm-up",
                          "params": {op: {k: v[k] for k in ("ctas_per_sm", "resolver")} for op, v in r["tuning"].items()},
                          "sweep_ms": {op: v["sweep_ms"] for op, v in r["tuning"].items()}}
    if r["ref_cuda"] is not None:
        rc = r["ref_cuda"]
        if "noa" in rc:  # set beside this run's own per-operation times
            mine_abs = {k: t for k, t in abs_ms.items() if k in FIVE}
            rc["cortado_b200_ms"] = {"noa": {k: op_ms[k] for k in FIVE}, "abs": mine_abs,
                                     "noa_reference_style": {k: r["ref_style"][k] for k in FIVE}}
            rc["speedup_sum_of_ops"] = {"noa": rc["noa"]["sum_ms"] / sum(op_ms[k] for k in FIVE),
                                        "abs": rc["abs"]["sum_ms"] / sum(mine_abs.values())}
        line["ref_cuda"] = rc
    if extras and world == 1:
        from cortado_b200.ops import Codec
        dev = torch.device("cuda", 0)

        def extra(key, fn):
            # a failing configuration is reported in its key; the line (and
            # the measured flow above) still prints
            try:
                line[key] = fn()
            except Exception as e:  # noqa: BLE001
                line[key] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.empty_cache()

        def with_codec(fn):
            c = Codec(0)
            try:
                return fn(c)
            finally:
                c.close()

        if "batched" in extras:
            extra("batched", lambda: with_codec(
                lambda c: bench_batched(c, dev, n_fields=args.batched_fields, max_mb=args.batched_max_mb)))
        if "serving" in extras:
            extra("serving", lambda: bench_serving(dev))
        if "chain" in extras:
            extra("chain", lambda: with_codec(lambda c: bench_chain(c, dev)))
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(r["x_host"])
    print(json.dumps(line))


if __name__ == "__main__":
    main()
