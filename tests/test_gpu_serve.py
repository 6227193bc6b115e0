"""Continuous-batching server: every request's result (its init or residual
stream) and every client's final reconstruction are identical when the trace
is served batched and overlapped (Server.run) and when each request runs alone
through the plain per-request pipeline (Server.run_plain); p50/p99 latencies
are reported.  Served at a Poisson rate and as a backlog (every request queued
at the start, small batches, so admission passes held-back clients)."""
import numpy as np
import pytest
import torch

from cortado_b200 import fields, storage
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _stream_len(buf: torch.Tensor) -> int:
    """Bytes of the stream at the start of an output buffer: header, size
    table and payloads (the buffer's capacity beyond that is not written)."""
    h = buf[:16].cpu().numpy()
    n = int(h[:8].view(np.int64)[0])
    chunks = -(-n // 16384)
    table = buf[16:16 + 2 * chunks].cpu().numpy().view(np.uint16)
    return 16 + 2 * chunks + int(table.astype(np.int64).sum())


def _server(dev_index, max_batch=16):
    from cortado_b200.serve import Server
    srv = Server(dev_index, mem_cap_bytes=4 * 10**9, max_inflight=16, n_streams=3, max_batch=max_batch)
    gens = {"a": fields.mixed_field(262144, "sinusoid", 1), "b": fields.mixed_field(1000000, "grf", 2),
            "c": fields.mixed_field(500001, "white", 3)}
    ranges = {}
    for name, x in gens.items():
        x = x.cuda()
        rng = float(x.max() - x.min())
        ranges[name] = rng
        srv.add_field(name, x, [float(storage.noa_scale(e, rng)) for e in (1e-1, 1e-3, 1e-5, 1e-7)])
    return srv, ranges


@pytest.mark.parametrize("backlog,max_batch", [(False, 16), (True, 4)])
def test_served_results_equal_alone(cuda_device, backlog, max_batch):
    from cortado_b200.serve import poisson_trace
    srv, ranges = _server(cuda_device.index, max_batch)
    rng = np.random.Generator(np.random.PCG64(11))
    trace = poisson_trace(rng, srv.fields, 60, rate_hz=20000.0, n_clients=4, ranges=ranges)
    if backlog:  # every request queued at the start: batches of 4, clients passing each other
        for r in trace:
            r.arrival = 0.0
    stats_b, out_b = srv.run(trace, keep_outputs=True)
    recon_b = {k: v["recon"].clone() for k, v in srv.clients.items()}
    bounds_b = {k: v["bound"] for k, v in srv.clients.items()}
    srv.reset_clients()
    for r in trace:
        r.done = -1.0
    stats_p, out_p = srv.run_plain(trace, keep_outputs=True)
    assert stats_b["requests"] == stats_p["requests"] == len(trace)
    for r in trace:
        a, b = out_b[r.rid], out_p[r.rid]
        n = _stream_len(b)
        assert _stream_len(a) == n and torch.equal(a[:n], b[:n]), r
    for k, v in srv.clients.items():
        assert bounds_b[k] == v["bound"]
        assert torch.equal(recon_b[k].view(torch.int32), v["recon"].view(torch.int32)), k
        x = srv.fields[k[1]].x
        assert O.maxabs(v["recon"].cpu().numpy(), x.cpu().numpy(), v["bound"]) == -1
    assert stats_b["p50_ms"] is not None and stats_b["p99_ms"] >= stats_b["p50_ms"]
    srv.close()


def test_memory_cap_spills_and_reloads_with_identical_results(cuda_device, tmp_path):
    """A cap below the working set: idle reconstructions and stored fields are
    spilled to host files and read back; every request's stream and every
    final reconstruction equal those of a server without the cap."""
    from cortado_b200.ops import max_stream_bytes
    from cortado_b200.serve import Server, poisson_trace
    big, ranges = _server(cuda_device.index, max_batch=4)
    rng = np.random.Generator(np.random.PCG64(23))
    trace = poisson_trace(rng, big.fields, 40, rate_hz=20000.0, n_clients=4, ranges=ranges)
    for r in trace:
        r.arrival = 0.0
    _, out_big = big.run(trace, keep_outputs=True)
    recon_big = {k: v["recon"].clone() for k, v in big.clients.items()}
    # room for the largest field's stored streams plus four output buffers and
    # four reconstructions of the largest field
    nmax = max(f.n_bytes for f in big.fields.values())
    cap = max(f.stored_total for f in big.fields.values()) + 4 * (max_stream_bytes(nmax) + nmax)
    small = Server(cuda_device.index, mem_cap_bytes=cap, max_inflight=16, n_streams=3, max_batch=4,
                   spill_dir=str(tmp_path))
    for name, f in big.fields.items():
        small.add_field(name, f.x, f.store_bounds, vrange=ranges[name])
    for r in trace:
        r.done = -1.0
    stats, out_small = small.run(trace, keep_outputs=True)
    assert stats["requests"] == len(trace) and stats["spills"] > 0 and stats["reloads"] > 0
    for r in trace:
        a, b = out_small[r.rid], out_big[r.rid]
        n = _stream_len(b)
        assert _stream_len(a) == n and torch.equal(a[:n], b[:n]), r
    for k, v in recon_big.items():
        st = small.clients[k]
        got = st["recon"] if st["recon"] is not None else torch.from_numpy(np.fromfile(st["spilled"], np.float32))
        assert torch.equal(got.cpu().view(torch.int32), v.cpu().view(torch.int32)), k
    small.close()
    big.close()
