"""The batched form (cortado_batch): one launch over many streams of uneven
sizes must produce exactly what one call per stream produces, for every
operation, including partial last chunks and one-chunk fields."""
import pytest
import torch

from cortado_b200 import fields, storage

pytestmark = pytest.mark.gpu

SIZES = [4096 * 4, 7 * 16384 + 4 * 333, 123 * 4, 16384 * 40, 5 * 16384 + 4, 3 * 16384]


@pytest.fixture(scope="module")
def codec(cuda_device):
    from cortado_b200.ops import Codec
    c = Codec(0)
    yield c
    c.close()


def _fields(dev):
    out = []
    for i, n in enumerate(SIZES):
        kind = ("sinusoid", "white", "grf")[i % 3]
        out.append(fields.mixed_field(n // 4, kind, seed=100 + i).to(dev))
    return out


def test_batch_all_ops_match_single_calls(codec, cuda_device):
    from cortado_b200.ops import max_stream_bytes
    xs = _fields(cuda_device)
    ebs = [float(storage.noa_scale(e, float(x.max() - x.min()))) for x, e in zip(xs, [1e-3, 1e-5, 1e-2, 1e-4, 1e-6, 1e-3])]
    # single calls
    stor1 = [codec.store(x, eb) for x, eb in zip(xs, ebs)]
    init1 = [codec.init_send(s, eb * 10) for s, eb in zip(stor1, ebs)]
    cl1 = [codec.init_recv(s) for s in init1]
    resi1 = [codec.resi_send(s, eb * 10, eb * 2) for s, eb in zip(stor1, ebs)]
    fin1 = [codec.resi_recv(c, r) for c, r in zip(cl1, resi1)]
    dec1 = [codec.store_decode(s) for s in stor1]

    sizes = torch.zeros(len(xs), dtype=torch.int64, device=cuda_device)

    def bufs(kind):
        if kind == "stream":
            return [torch.empty(max_stream_bytes(x.numel() * 4), dtype=torch.uint8, device=cuda_device) for x in xs]
        return [torch.empty_like(x) for x in xs]

    def trim(outs):
        torch.cuda.synchronize()
        codec.sync()
        return [o[: int(sizes[i].item())] for i, o in enumerate(outs)]

    out = bufs("stream")
    codec.batch("store", [dict(**{"in": x}, out=o, out_size=sizes[i:i + 1], n_bytes=x.numel() * 4, eb1=eb)
                          for i, (x, o, eb) in enumerate(zip(xs, out, ebs))])
    stor2 = trim(out)
    assert all(torch.equal(a, b) for a, b in zip(stor1, stor2))

    out = bufs("stream")
    codec.batch("init_send", [dict(**{"in": s}, out=o, out_size=sizes[i:i + 1], n_bytes=x.numel() * 4, eb1=eb * 10)
                              for i, (s, x, o, eb) in enumerate(zip(stor1, xs, out, ebs))])
    assert all(torch.equal(a, b) for a, b in zip(init1, trim(out)))

    out = bufs("stream")
    codec.batch("resi_send", [dict(**{"in": s}, out=o, out_size=sizes[i:i + 1], n_bytes=x.numel() * 4, eb1=eb * 10,
                                   eb2=eb * 2) for i, (s, x, o, eb) in enumerate(zip(stor1, xs, out, ebs))])
    assert all(torch.equal(a, b) for a, b in zip(resi1, trim(out)))

    for op, ins, ref in (("init_recv", init1, cl1), ("store_decode", stor1, dec1)):
        out = bufs("floats")
        codec.batch(op, [dict(**{"in": s}, out=o, out_size=sizes[i:i + 1], n_bytes=x.numel() * 4)
                         for i, (s, x, o) in enumerate(zip(ins, xs, out))])
        torch.cuda.synchronize()
        codec.sync()
        assert all(torch.equal(a.view(torch.int32), b.view(torch.int32)) for a, b in zip(ref, out)), op

    out = bufs("floats")
    codec.batch("resi_recv", [dict(**{"in": r}, src=c, out=o, out_size=sizes[i:i + 1], n_bytes=x.numel() * 4)
                              for i, (r, c, x, o) in enumerate(zip(resi1, cl1, xs, out))])
    torch.cuda.synchronize()
    codec.sync()
    assert all(torch.equal(a.view(torch.int32), b.view(torch.int32)) for a, b in zip(fin1, out))


def test_batch_rejects_bad_items(codec, cuda_device):
    from cortado_b200._native import CortadoError
    x = torch.zeros(1024, device=cuda_device)
    out = torch.empty(100, dtype=torch.uint8, device=cuda_device)
    size = torch.zeros(1, dtype=torch.int64, device=cuda_device)
    with pytest.raises(CortadoError) as e:
        codec.batch("store", [dict(**{"in": x}, out=out, out_size=size, n_bytes=4096, eb1=1e-3)])
    assert e.value.name == "CAPACITY"


def test_batch_groups_on_one_input_match_single_calls(codec, cuda_device):
    """Adjacent items of an encoder's batch that read the same input (one field
    stored at several bounds, one stored stream sent at several, plain and
    applied to clients, the serving loop's and the many-bounds store's
    pattern): every stream and every client reconstruction must equal its
    single call, for one-chunk, partial-chunk and many-chunk inputs next to
    items on other inputs."""
    from cortado_b200.ops import max_stream_bytes
    xs = _fields(cuda_device)
    a, b, one = xs[1], xs[3], xs[0]  # 7 chunks + a partial one; 40 chunks; exactly one chunk
    plan = [(a, 1e-2), (a, 1e-3), (a, 1e-5), (b, 1e-4), (one, 1e-3), (one, 1e-6), (a, 1e-4), (b, 1e-2),
            (b, 1e-6), (b, 1e-3)]
    ebs = [float(storage.noa_scale(e, float(x.max() - x.min()))) for x, e in plan]
    sizes = torch.zeros(len(plan), dtype=torch.int64, device=cuda_device)

    def run(op, items):
        codec.batch(op, items)
        torch.cuda.synchronize()
        codec.sync()

    ref = [codec.store(x, eb) for (x, _), eb in zip(plan, ebs)]
    outs = [torch.empty(max_stream_bytes(x.numel() * 4), dtype=torch.uint8, device=cuda_device) for x, _ in plan]
    run("store", [dict(**{"in": x}, out=o, out_size=sizes[i:i + 1], n_bytes=x.numel() * 4, eb1=eb)
                  for i, ((x, _), o, eb) in enumerate(zip(plan, outs, ebs))])
    for i, r in enumerate(ref):
        assert torch.equal(outs[i][: int(sizes[i].item())], r), i

    # one stored stream per input, each sent at three bounds (and one lone item)
    sends = []
    for x, s, eb in ((a, ref[2], ebs[2]), (b, ref[8], ebs[8]), (one, ref[5], ebs[5])):
        sends += [(x, s, eb * 1000, eb * 10), (x, s, eb * 100, eb * 10), (x, s, eb * 10, eb * 2)]
    sends.append((a, ref[1], ebs[1] * 10, ebs[1] * 2))
    n = len(sends)
    sizes = torch.zeros(n, dtype=torch.int64, device=cuda_device)
    streams = [torch.empty(max_stream_bytes(x.numel() * 4), dtype=torch.uint8, device=cuda_device) for x, *_ in sends]
    init_ref = [codec.init_send(s, e1) for _, s, e1, _ in sends]
    resi_ref = [codec.resi_send(s, e1, e2) for _, s, e1, e2 in sends]

    run("init_send", [dict(**{"in": s}, out=o, out_size=sizes[i:i + 1], n_bytes=x.numel() * 4, eb1=e1)
                      for i, ((x, s, e1, _), o) in enumerate(zip(sends, streams))])
    for i, r in enumerate(init_ref):
        assert torch.equal(streams[i][: int(sizes[i].item())], r), ("init_send", i)
    run("resi_send", [dict(**{"in": s}, out=o, out_size=sizes[i:i + 1], n_bytes=x.numel() * 4, eb1=e1, eb2=e2)
                      for i, ((x, s, e1, e2), o) in enumerate(zip(sends, streams))])
    for i, r in enumerate(resi_ref):
        assert torch.equal(streams[i][: int(sizes[i].item())], r), ("resi_send", i)

    # the fused forms: every member writes its own client's reconstruction
    clients = [torch.full_like(x, 7.0) for x, *_ in sends]
    run("init_send_apply", [dict(**{"in": s}, src=c, out=o, out_size=sizes[i:i + 1], n_bytes=x.numel() * 4, eb1=e1)
                            for i, ((x, s, e1, _), o, c) in enumerate(zip(sends, streams, clients))])
    for i, r in enumerate(init_ref):
        assert torch.equal(streams[i][: int(sizes[i].item())], r), ("init_send_apply", i)
        assert torch.equal(clients[i].view(torch.int32), codec.init_recv(r).view(torch.int32)), ("init client", i)
    before = [c.clone() for c in clients]
    run("resi_send_apply", [dict(**{"in": s}, src=c, out=o, out_size=sizes[i:i + 1], n_bytes=x.numel() * 4,
                                 eb1=e1, eb2=e2)
                            for i, ((x, s, e1, e2), o, c) in enumerate(zip(sends, streams, clients))])
    for i, r in enumerate(resi_ref):
        assert torch.equal(streams[i][: int(sizes[i].item())], r), ("resi_send_apply", i)
        assert torch.equal(clients[i].view(torch.int32), codec.resi_recv(before[i], r).view(torch.int32)), \
            ("resi client", i)
