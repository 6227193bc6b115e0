"""init_send / resi_send fused with the client's receive (cortado_*_send_apply
and the batched CORTADO_OP_*_SEND_APPLY): the stream is byte-identical to the
separate send's and the client's reconstruction bit-identical to the separate
receive of that stream, and both equal the oracle's, on fields with partial
last chunks, lossless outliers, infinities, and incompressible chunks (raw
init chunks, whose bins init_recv emits unchanged)."""
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


def _cases():
    rng = np.random.Generator(np.random.PCG64(77))
    out = []
    x = fields.mixed_field(9 * 4096 + 321, "sinusoid", 5).numpy()
    out.append(("sinusoid", x, 1e-3))
    w = fields.mixed_field(6 * 4096, "white", 6).numpy()
    out.append(("white_fine", w, 1e-7))  # incompressible: raw chunks
    y = rng.normal(0, 1, 5 * 4096 + 17).astype(np.float32)
    idx = rng.choice(y.size, 40, replace=False)
    y[idx] = rng.choice([-1.0, 1.0], 40).astype(np.float32) * 1e6
    y[idx[:2]] = [np.inf, -np.inf]
    out.append(("outliers", y, 1e-4))
    b = (rng.integers(0, 2**23, 3 * 4096, dtype=np.uint32) | (rng.integers(100, 140, 3 * 4096, dtype=np.uint32) << 23))
    out.append(("randbits", b.view(np.float32), 1e-2))
    return out


def u8(t):
    return bytes(t.cpu().numpy())


def bits(t):
    a = t.cpu().numpy() if isinstance(t, torch.Tensor) else t
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("name,x,eb", _cases(), ids=[c[0] for c in _cases()])
def test_send_apply_equals_send_then_receive(codec, name, x, eb):
    from cortado_b200.ops import max_stream_bytes
    xg = torch.from_numpy(x).cuda()
    n = x.size * 4
    stor = codec.store(xg, eb)
    stor_o = O.store_encode(x, eb)
    assert u8(stor) == stor_o
    cap = max_stream_bytes(n)
    sz = torch.zeros(2, dtype=torch.int64, device="cuda")
    for req in (eb * 10, eb * 3, eb):
        init = torch.empty(cap, dtype=torch.uint8, device="cuda")
        client = torch.full_like(xg, 7.0)
        codec.s2c_encode_apply(stor, init, sz[0:1], req, n, client)
        codec.sync()
        init_ref = codec.init_send(stor, req)
        assert u8(init[: int(sz[0].item())]) == u8(init_ref) == O.init_send(stor_o, req), req
        assert np.array_equal(bits(client), bits(codec.init_recv(init_ref))), req
        assert np.array_equal(bits(client), bits(O.init_recv(O.init_send(stor_o, req)))), req
        for dst in (req / 4, req / 100):
            if dst < eb:
                continue
            resi = torch.empty(cap, dtype=torch.uint8, device="cuda")
            before = client.clone()
            codec.residual_encode_apply(stor, resi, sz[1:2], req, dst, n, client)
            codec.sync()
            resi_ref = codec.resi_send(stor, req, dst)
            assert u8(resi[: int(sz[1].item())]) == u8(resi_ref), (req, dst)
            assert np.array_equal(bits(client), bits(codec.resi_recv(before, resi_ref))), (req, dst)
            assert np.array_equal(bits(client), bits(O.resi_recv(bits(before).view(np.float32), u8(resi_ref))))
            client.copy_(before)


def test_batched_send_apply_equals_single(codec, cuda_device):
    from cortado_b200.ops import max_stream_bytes
    cases = _cases()
    xs = [torch.from_numpy(x).cuda() for _, x, _ in cases]
    ebs = [eb for _, _, eb in cases]
    stors = [codec.store(x, eb) for x, eb in zip(xs, ebs)]
    sizes = torch.zeros(len(xs), dtype=torch.int64, device=cuda_device)
    outs = [torch.empty(max_stream_bytes(x.numel() * 4), dtype=torch.uint8, device=cuda_device) for x in xs]
    clients = [torch.zeros_like(x) for x in xs]
    codec.batch("init_send_apply", [dict(**{"in": s}, out=o, out_size=sizes[i:i + 1], n_bytes=x.numel() * 4,
                                         eb1=eb * 10, src=cl)
                                    for i, (s, x, o, eb, cl) in enumerate(zip(stors, xs, outs, ebs, clients))])
    torch.cuda.synchronize()
    codec.sync()
    for i, (s, eb) in enumerate(zip(stors, ebs)):
        ref = codec.init_send(s, eb * 10)
        assert u8(outs[i][: int(sizes[i].item())]) == u8(ref)
        assert torch.equal(clients[i].view(torch.int32), codec.init_recv(ref).view(torch.int32))
    before = [c.clone() for c in clients]
    codec.batch("resi_send_apply", [dict(**{"in": s}, out=o, out_size=sizes[i:i + 1], n_bytes=x.numel() * 4,
                                         eb1=eb * 10, eb2=eb * 2, src=cl)
                                    for i, (s, x, o, eb, cl) in enumerate(zip(stors, xs, outs, ebs, clients))])
    torch.cuda.synchronize()
    codec.sync()
    for i, (s, eb) in enumerate(zip(stors, ebs)):
        ref = codec.resi_send(s, eb * 10, eb * 2)
        assert u8(outs[i][: int(sizes[i].item())]) == u8(ref)
        assert torch.equal(clients[i].view(torch.int32), codec.resi_recv(before[i], ref).view(torch.int32))
