"""Oracle parity on exactly the configurations bench.py times.

Every stream is compared byte for byte with the CPU oracle and every decoded
float bit for bit, on the benchmark's own fields and bounds:

* the headline flow on the 512^3 sinusoid + noise + 0.1% +-1e6 outliers field
  (NOA store 1e-4, init 1e-2, residual 1e-2 -> 1e-4), the same field's ABS
  flow (store 1e-6, init 1e-3, residual 1e-3 -> 1e-5) and the NOA flow on
  the generator without the outliers (bounds scaled on the device too);
* the progressive chain on the 16384^2 GRF (k^-2.5): the four stored streams,
  the init stream and the five residual streams of the captured graph's
  replay, and every reconstruction;
* a subset of the many-fields configuration (fields of 1-256 MiB, all three
  generators, 4 NOA bounds each), each batched item against the oracle;
* a served trace: every request's stream and every client's final
  reconstruction against the oracle.

Reference counterparts of the compared operations: include/d_server_encode.h:51-143,
include/d_s2c.h:51-200, include/d_client_encode.h:173-259,
include/d_residual_encode.h:51-347."""
import numpy as np
import pytest
import torch

from cortado_b200 import fields, storage
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def codec(cuda_device):
    from cortado_b200.ops import Codec
    c = Codec(0)
    yield c
    c.close()


def u8(t: torch.Tensor) -> bytes:
    return bytes(t.cpu().numpy())


def bits(a) -> np.ndarray:
    if isinstance(a, torch.Tensor):
        a = a.cpu().numpy()
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def field_512(cuda_device):
    import bench
    x = bench.make_field(2, cuda_device)  # the benchmark's own field (seed 2, 512^3)
    return x, x.cpu().numpy()


def _flow(codec, x, xn, eb_store, eb_src, eb_dst):
    """The benchmark step's five operations, each compared with the oracle."""
    stor = codec.store(x, eb_store)
    stor_o = O.store_encode(xn, eb_store)
    assert u8(stor) == stor_o, "store"
    init = codec.init_send(stor, eb_src)
    init_o = O.init_send(stor_o, eb_src)
    assert u8(init) == init_o, "init_send"
    cl = codec.init_recv(init)
    cl_o = O.init_recv(init_o)
    assert np.array_equal(bits(cl), bits(cl_o)), "init_recv"
    resi = codec.resi_send(stor, eb_src, eb_dst)
    resi_o = O.resi_send(stor_o, eb_src, eb_dst)
    assert u8(resi) == resi_o, "resi_send"
    fin = codec.resi_recv(cl, resi)
    fin_o = O.resi_recv(cl_o, resi_o)
    assert np.array_equal(bits(fin), bits(fin_o)), "resi_recv"
    assert O.maxabs(fin_o, xn, eb_dst) == -1
    assert O.maxabs(cl_o, xn, eb_src) == -1
    return len(stor_o), len(init_o), len(resi_o)


def test_headline_noa_flow_512_matches_oracle(codec, field_512):
    import bench
    x, xn = field_512
    lo, hi = codec.INOA_find_range(x)
    rng = storage.value_range(lo, hi)
    assert rng == O.noa_range(xn)
    ebs = [float(storage.noa_scale(e, rng)) for e in (bench.EB_STORE, bench.EB_SRC, bench.EB_DST)]
    sizes = _flow(codec, x, xn, *ebs)
    assert sizes[0] < len(xn) * 4  # compresses


def test_abs_flow_512_matches_oracle(codec, field_512):
    import bench
    x, xn = field_512
    ebs = [float(storage.f32(e)) for e in (bench.ABS_STORE, bench.ABS_SRC, bench.ABS_DST)]
    _flow(codec, x, xn, *ebs)


def test_no_outlier_noa_flow_512_matches_oracle(codec, cuda_device):
    """The bench's no-outlier flow: the same generator without the outliers
    at 512^3, the same NOA bounds, the bounds scaled on the device."""
    import bench
    x = bench.make_field(2, cuda_device, outliers=False)
    xn = x.cpu().numpy()
    mm = codec.INOA_find_range_device(x)
    rng = O.noa_range(xn)
    assert storage.value_range(*mm.cpu().tolist()) == rng
    ebs = [float(storage.noa_scale(e, rng)) for e in (bench.EB_STORE, bench.EB_SRC, bench.EB_DST)]
    sizes = _flow(codec, x, xn, *ebs)
    n = x.numel() * 4
    # the device-scaled entry points write the same streams
    from cortado_b200.ops import max_stream_bytes
    sz = torch.zeros(3, dtype=torch.int64, device=cuda_device)
    stor = torch.empty(max_stream_bytes(n), dtype=torch.uint8, device=cuda_device)
    init = torch.empty_like(stor)
    resi = torch.empty_like(stor)
    codec.server_encode_noa(x, n, stor, sz[0:1], mm, float(storage.f32(bench.EB_STORE)))
    codec.s2c_encode_noa(stor, init, sz[1:2], mm, float(storage.f32(bench.EB_SRC)), n)
    codec.residual_encode_noa(stor, resi, sz[2:3], mm, float(storage.f32(bench.EB_SRC)),
                              float(storage.f32(bench.EB_DST)), n)
    codec.sync()
    assert sz.cpu().tolist() == [sizes[0], sizes[1], sizes[2]]
    assert u8(stor[:sizes[0]]) == O.store_encode(xn, ebs[0])


def test_chain_16384_graph_streams_match_oracle(codec, cuda_device):
    """The benchmark's progressive chain (bench_chain): stored at NOA
    1e-1/1e-3/1e-5/1e-7, init 1e-1, residual steps to 1e-2 ... 1e-6, replayed
    from the captured graph."""
    from cortado_b200.chain import ProgressiveChain
    x = fields.grf((16384, 16384), 4, slope=2.5, device=cuda_device).reshape(-1)
    lo, hi = codec.INOA_find_range(x)
    rng = storage.value_range(lo, hi)
    nb = lambda e: float(storage.noa_scale(e, rng))  # noqa: E731
    ch = ProgressiveChain(codec, x, [nb(e) for e in (1e-1, 1e-3, 1e-5, 1e-7)], nb(1e-1),
                          [nb(e) for e in (1e-2, 1e-3, 1e-4, 1e-5, 1e-6)])
    ch.capture()
    for r in ch.recon:
        r.zero_()
    ch.replay()
    torch.cuda.synchronize()
    codec.sync()
    assert (ch.first_bad == -1).all()
    xn = x.cpu().numpy()
    del x
    stored_o = []
    for buf, n, eb in zip(ch.stored, ch.stored_bytes, ch.store_bounds):
        s = O.store_encode(xn, eb)
        assert u8(buf[:n]) == s, ("store", eb)
        stored_o.append(s)
    sizes = [int(v) for v in ch.stream_sizes.tolist()]
    prev = None
    for j, eb in enumerate(ch.bounds):
        src = stored_o[ch.sel[j]]
        if j == 0:
            s_o = O.init_send(src, eb)
            r_o = O.init_recv(s_o)
        else:
            s_o = O.resi_send(src, ch.bounds[j - 1], eb)
            r_o = O.resi_recv(prev, s_o)
        assert sizes[j] == len(s_o) and u8(ch.streams[j][: sizes[j]]) == s_o, ("stream", j)
        assert np.array_equal(bits(ch.recon[j]), bits(r_o)), ("recon", j)
        assert O.maxabs(r_o, xn, eb) == -1
        prev = r_o
    del ch


def test_batched_store_subset_matches_oracle(codec, cuda_device):
    """Eight fields of the many-fields configuration (spanning its sizes and
    all three generators), each stored at NOA 1e-1 ... 1e-4 in one batched
    launch; every item's stream equals the oracle's."""
    from cortado_b200.ops import max_stream_bytes
    specs = fields.field_set(64, 3, 1 << 20, 256 << 20)
    order = sorted(range(len(specs)), key=lambda i: specs[i][0])
    pick = sorted({order[k] for k in (0, 9, 18, 27, 36, 45, 54, 63)})
    kinds = {specs[i][1] for i in pick}
    for i in order:  # make every generator appear
        if specs[i][1] not in kinds:
            pick.append(i)
            kinds.add(specs[i][1])
    bounds = ("1e-1", "1e-2", "1e-3", "1e-4")
    xs = [fields.mixed_field(*specs[i], device=cuda_device) for i in pick]
    items, want = [], []
    sizes = torch.zeros(len(xs) * len(bounds), dtype=torch.int64, device=cuda_device)
    for i, x in enumerate(xs):
        xn = x.cpu().numpy()
        r = O.noa_range(xn)
        for j, b in enumerate(bounds):
            k = i * len(bounds) + j
            eb = float(storage.noa_scale(b, r))
            out = torch.empty(max_stream_bytes(x.numel() * 4), dtype=torch.uint8, device=cuda_device)
            items.append(dict(**{"in": x}, out=out, out_size=sizes[k:k + 1], n_bytes=x.numel() * 4, eb1=eb))
            want.append(O.store_encode(xn, eb))
    codec.batch("store", items)
    torch.cuda.synchronize()
    codec.sync()
    got = sizes.tolist()
    for k, (it, w) in enumerate(zip(items, want)):
        assert got[k] == len(w) and u8(it["out"][: got[k]]) == w, k


def test_served_trace_matches_oracle(cuda_device):
    """A trace of the serving configuration's mix (60% init at NOA 1e-1 ..
    1e-3, 40% residual 1-3 decades finer) on resident fields of 4-48 MiB,
    served with continuous batching; every request's stream and every
    client's final reconstruction equal the oracle's, replayed in each
    client's order."""
    from cortado_b200.serve import Server, poisson_trace
    rng = np.random.Generator(np.random.PCG64(5))
    srv = Server(cuda_device.index, mem_cap_bytes=8 * 10**9, max_inflight=32, n_streams=3, max_batch=8)
    ranges, xs, stored_o = {}, {}, {}
    for i, spec in enumerate(fields.field_set(6, 5, 4 << 20, 48 << 20, rng=rng)):
        x = fields.mixed_field(*spec, device=cuda_device)
        xn = x.cpu().numpy()
        r = O.noa_range(xn)
        name = f"f{i}"
        ranges[name], xs[name] = float(r), xn
        srv.add_field(name, x, [float(storage.noa_scale(e, r)) for e in (1e-1, 1e-3, 1e-5, 1e-7)])
        f = srv.fields[name]
        stored_o[name] = [O.store_encode(xn, eb) for eb in f.store_bounds]
        for s, so in zip(f.stored, stored_o[name]):
            assert u8(s) == so
    trace = poisson_trace(rng, srv.fields, 80, rate_hz=20000.0, n_clients=4, ranges=ranges)
    _, outs = srv.run(trace, keep_outputs=True)
    cur = {}
    for r in sorted(trace, key=lambda r: r.arrival):
        f = srv.fields[r.field]
        i = storage.select_stored([storage.f32(e) for e in f.store_bounds], r.bound)
        key = (r.client, r.field)
        if r.kind == "init":
            s_o = O.init_send(stored_o[r.field][i], r.bound)
            rec = O.init_recv(s_o)
        else:
            src_bound, prev = cur[key]
            s_o = O.resi_send(stored_o[r.field][i], src_bound, r.bound)
            rec = O.resi_recv(prev, s_o)
        assert u8(outs[r.rid][: len(s_o)]) == s_o, r
        cur[key] = (r.bound, rec)
    for key, (bound, rec) in cur.items():
        st = srv.clients[key]
        assert st["bound"] == bound
        assert np.array_equal(bits(st["recon"]), bits(rec)), key
        assert O.maxabs(rec, xs[key[1]], bound) == -1
    srv.close()
