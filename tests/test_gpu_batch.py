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
