"""Admission logic of the continuous-batching server (Server.run), on the CPU:
the GPU launches are replaced by fakes whose completion events report done
after a few polls.  Checked: a client's steps on a field start only after its
previous step finished and in arrival order; batches hold at most max_batch
requests; at most max_inflight requests (and, when set, max_batches batches)
are in flight; the memory cap holds,
counting reconstructions and pooled output buffers; a client held back by its
own running step does not hold back other clients; idle state is spilled to
host files and read back unchanged; a request larger than the memory cap is
an error, not a hang."""
import numpy as np
import pytest
import torch

from cortado_b200 import serve
from cortado_b200.ops import max_stream_bytes


class _Event:
    def __init__(self, polls):
        self.polls = polls

    def query(self):
        self.polls -= 1
        return self.polls < 0


class _Codec:
    def sync(self, stream=None):
        pass


def _server(sizes, max_inflight, max_batch, mem_cap, polls=3, stored_bytes=0, spill_dir=None, max_batches=None):
    srv = serve.Server.__new__(serve.Server)
    srv.dev = torch.device("cpu")
    srv.codecs = [_Codec() for _ in range(3)]
    srv.streams = [None] * 3
    srv.mem_cap = mem_cap
    srv.max_inflight = max_inflight
    srv.max_batch = max_batch
    srv.max_batches = max_batches
    srv.fields = {name: serve.Field(name, torch.zeros(n // 4), [1.0]) for name, n in sizes.items()}
    srv.clients = {}
    srv.mem_used = 0
    srv._free_out = {}
    srv.spill_dir = spill_dir
    srv.spills = srv.reloads = srv._tick = 0
    for f in srv.fields.values():  # one fake stored stream per field
        f.stored = [torch.arange(stored_bytes, dtype=torch.int64).to(torch.uint8)] if stored_bytes else []
        f.stored_bytes = [stored_bytes] if stored_bytes else []
        srv.mem_used += stored_bytes
    launches, launched, batches = [], [], []
    recon_of = {}

    def fake_launch(k, reqs):
        launched.extend(reqs)
        outs = {r.rid: srv._out_buffer(srv.fields[r.field]) for r in reqs}
        for r in reqs:  # the batch's use of its resident state
            st = srv.clients[(r.client, r.field)]
            assert st["recon"] is not None and srv.fields[r.field].spilled is None
            if r.kind == "resi" and st["bound"] is not None:  # a spilled client comes back as it left
                assert torch.equal(st["recon"], recon_of[(r.client, r.field)])
            st["recon"].fill_(float(r.rid))  # a client's state changes with each step
            recon_of[(r.client, r.field)] = st["recon"].clone()
            st["bound"] = r.bound
        launches.append({"stream": k, "rids": [r.rid for r in reqs],
                         "inflight": sum(1 for r in launched if r.done < 0),
                         "batches_inflight": sum(1 for b in batches if any(r.done < 0 for r in b)),
                         "mem_used": srv.mem_used,
                         "prev_done": [all(p.done >= 0 for p in launched[:-len(reqs)]
                                           if (p.client, p.field) == (r.client, r.field)) for r in reqs]})
        batches.append(list(reqs))
        return _Event(polls), outs, None

    srv._launch = fake_launch
    return srv, launches


def _trace(rng, names, n, n_clients, rate_hz):
    reqs, t = [], 0.0
    for rid in range(n):
        if rate_hz:
            t += rng.exponential(1.0 / rate_hz)
        reqs.append(serve.Request(rid, "init" if rng.random() < 0.6 else "resi", int(rng.integers(n_clients)),
                                  names[int(rng.integers(len(names)))], 1e-3, t))
    return reqs


@pytest.mark.parametrize("rate_hz", [None, 5e4])
@pytest.mark.parametrize("max_batch,max_inflight", [(1, 4), (4, 8), (16, 64)])
def test_admission_invariants(rate_hz, max_batch, max_inflight):
    rng = np.random.Generator(np.random.PCG64(3))
    sizes = {f"f{i}": int(rng.integers(1, 64)) << 16 for i in range(6)}
    cap = 5 * max(max_stream_bytes(n) for n in sizes.values())
    srv, launches = _server(sizes, max_inflight, max_batch, cap)
    trace = _trace(rng, sorted(sizes), 120, 3, rate_hz)
    stats, _ = srv.run(trace)
    assert stats["requests"] == len(trace)
    assert all(r.done >= r.arrival for r in trace)
    order = [rid for b in launches for rid in b["rids"]]
    assert sorted(order) == list(range(len(trace)))
    for b in launches:
        assert 1 <= len(b["rids"]) <= max_batch
        assert b["inflight"] <= max_inflight
        assert b["mem_used"] <= cap
        assert all(b["prev_done"])
    pos = {rid: i for i, rid in enumerate(order)}
    by_key = {}
    for r in trace:
        by_key.setdefault((r.client, r.field), []).append(r.rid)
    for rids in by_key.values():
        assert [pos[x] for x in rids] == sorted(pos[x] for x in rids)
    assert srv.mem_used == _accounted(srv)


@pytest.mark.parametrize("max_batches", [1, 2])
@pytest.mark.parametrize("rate_hz", [None, 5e4])
def test_batches_in_flight_limit(rate_hz, max_batches):
    """With max_batches set, a batch is launched only while fewer batches are
    in flight, so the requests that arrive meanwhile gather into the next one."""
    rng = np.random.Generator(np.random.PCG64(4))
    sizes = {f"f{i}": int(rng.integers(1, 64)) << 16 for i in range(6)}
    srv, launches = _server(sizes, 64, 16, 10**12, max_batches=max_batches)
    trace = _trace(rng, sorted(sizes), 120, 8, rate_hz)
    stats, _ = srv.run(trace)
    assert stats["requests"] == len(trace)
    assert all(b["batches_inflight"] < max_batches for b in launches)
    assert sorted(rid for b in launches for rid in b["rids"]) == list(range(len(trace)))
    if rate_hz is None:  # everything queued: full batches but for the clients' own order
        assert max(len(b["rids"]) for b in launches) > 1


def _accounted(srv):
    """Device bytes the server holds: resident reconstructions, resident
    stored streams and pooled output buffers."""
    rec = sum(srv.fields[k[1]].n_bytes for k, st in srv.clients.items() if st["recon"] is not None)
    stor = sum(f.stored_total for f in srv.fields.values() if f.spilled is None)
    pool = sum(len(p) * max_stream_bytes(srv.fields[n].n_bytes) for n, p in srv._free_out.items())
    return rec + stor + pool


def test_held_client_does_not_block_others():
    sizes = {"a": 1 << 20, "b": 1 << 20}
    srv, launches = _server(sizes, 16, 16, 10**12)
    R = serve.Request
    trace = [R(0, "init", 0, "a", 1e-3, 0.0), R(1, "resi", 0, "a", 1e-4, 0.0), R(2, "init", 1, "a", 1e-3, 0.0),
             R(3, "init", 0, "b", 1e-3, 0.0), R(4, "resi", 0, "a", 1e-5, 0.0), R(5, "init", 2, "b", 1e-3, 0.0)]
    srv.run(trace)
    assert launches[0]["rids"] == [0, 2, 3, 5]
    assert [b["rids"] for b in launches[1:]] == [[1], [4]]


def test_new_client_reconstruction_counts_against_cap():
    """A first request of a client reserves its reconstruction: with room for
    the output stream but not for the reconstruction as well, the request
    cannot run (admission used to check the stream only)."""
    n = 1 << 20
    srv, _ = _server({"a": n}, 16, 16, max_stream_bytes(n) + n - 4)
    with pytest.raises(RuntimeError, match="memory cap"):
        srv.run([serve.Request(0, "init", 0, "a", 1e-3, 0.0)])
    srv, launches = _server({"a": n}, 16, 16, max_stream_bytes(n) + n)
    srv.run([serve.Request(0, "init", 0, "a", 1e-3, 0.0)])
    assert len(launches) == 1 and srv.mem_used == _accounted(srv) <= srv.mem_cap


def test_cap_spills_idle_state_and_reloads_it(tmp_path):
    """Under a cap that holds one field's stored stream, one client's
    reconstruction and one output buffer at a time, idle reconstructions and
    idle fields are written to host files (raw float32; a .stor.NN/.stor.meta
    storage directory) and read back, unchanged, when a request needs them
    (the fake launch checks a residual's client state)."""
    from cortado_b200 import storage
    n = sb = 1 << 18
    cap = max_stream_bytes(n) + n + sb + 3 * 4096
    srv, launches = _server({"a": n, "b": n}, 16, 4, cap, stored_bytes=sb, spill_dir=str(tmp_path))
    R = serve.Request
    trace = [R(0, "init", 0, "a", 1e-3, 0.0), R(1, "init", 1, "b", 1e-3, 0.0), R(2, "resi", 0, "a", 1e-4, 0.0),
             R(3, "resi", 1, "b", 1e-4, 0.0), R(4, "init", 2, "a", 1e-3, 0.0), R(5, "resi", 0, "a", 1e-5, 0.0)]
    stats, _ = srv.run(trace)
    assert stats["requests"] == len(trace) and all(r.done >= 0 for r in trace)
    assert stats["spills"] >= 4 and stats["reloads"] >= 3
    assert max(b["mem_used"] for b in launches) <= cap
    assert srv.mem_used == _accounted(srv) <= cap
    for f in srv.fields.values():
        if f.spilled is not None:  # the reference's storage layout
            meta = storage.read_storage_meta(f.spilled)
            assert meta.name == f.name and len(meta.ebs) == len(f.store_bounds)
            assert (tmp_path / "fields" / f.name / storage.stor_name(f.name, 0)).stat().st_size == sb


def test_request_over_memory_cap_raises():
    srv, _ = _server({"a": 1 << 20}, 16, 16, 1 << 10)
    with pytest.raises(RuntimeError, match="memory cap"):
        srv.run([serve.Request(0, "init", 0, "a", 1e-3, 0.0)])
