"""NOA bounds scaled on the device (cortado_noa_range_device and the
cortado_*_noa entry points, the fused send-and-apply forms included): the
streams and client reconstructions are byte-identical to the
host-scaled calls with the drivers' float arithmetic (storage.noa_scale of
the device range), bound errors are latched and written nowhere, and a whole
NOA flow is captured in a CUDA graph and replayed with identical results
(nothing in it waits for the host)."""
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


def _fields():
    rng = np.random.Generator(np.random.PCG64(91))
    y = rng.normal(0, 1, 7 * 4096 + 33).astype(np.float32)
    y[rng.choice(y.size, 30, replace=False)] = 1e6
    return [("sinusoid", fields.mixed_field(9 * 4096 + 5, "sinusoid", 2).numpy()),
            ("outliers", y), ("white", fields.mixed_field(4 * 4096, "white", 4).numpy())]


def u8(t):
    return bytes(t.cpu().numpy())


@pytest.mark.parametrize("name,x", _fields(), ids=[n for n, _ in _fields()])
def test_device_noa_equals_host_scaled(codec, name, x):
    from cortado_b200.ops import max_stream_bytes
    xg = torch.from_numpy(x).cuda()
    n = x.size * 4
    mm = codec.INOA_find_range_device(xg)
    lo, hi = codec.INOA_find_range(xg)
    assert mm.cpu().tolist() == [lo, hi]
    rng = storage.value_range(lo, hi)
    cap = max_stream_bytes(n)
    sz = torch.zeros(4, dtype=torch.int64, device="cuda")
    for store_noa in (1e-1, 1e-3, 1e-5, 1e-7):
        stor = torch.empty(cap, dtype=torch.uint8, device="cuda")
        codec.server_encode_noa(xg, n, stor, sz[0:1], mm, store_noa)
        codec.sync()
        ref = codec.store(xg, float(storage.noa_scale(store_noa, rng)))
        assert u8(stor[: int(sz[0].item())]) == u8(ref), store_noa
        req, dst = store_noa * 100, store_noa * 3
        init = torch.empty(cap, dtype=torch.uint8, device="cuda")
        codec.s2c_encode_noa(ref, init, sz[1:2], mm, req, n)
        resi = torch.empty(cap, dtype=torch.uint8, device="cuda")
        codec.residual_encode_noa(ref, resi, sz[2:3], mm, req, dst, n)
        codec.sync()
        ea, eb = float(storage.noa_scale(req, rng)), float(storage.noa_scale(dst, rng))
        assert u8(init[: int(sz[1].item())]) == u8(codec.init_send(ref, ea)) == O.init_send(u8(ref), ea)
        assert u8(resi[: int(sz[2].item())]) == u8(codec.resi_send(ref, ea, eb)) == O.resi_send(u8(ref), ea, eb)


@pytest.mark.parametrize("name,x", _fields(), ids=[n for n, _ in _fields()])
def test_fused_device_noa_equals_host_scaled(codec, name, x):
    """cortado_*_send_apply_noa: stream and client reconstruction equal the
    host-scaled fused calls' and the separate receive's."""
    from cortado_b200.ops import max_stream_bytes
    xg = torch.from_numpy(x).cuda()
    n = x.size * 4
    mm = codec.INOA_find_range_device(xg)
    rng = storage.value_range(*mm.cpu().tolist())
    cap = max_stream_bytes(n)
    sz = torch.zeros(4, dtype=torch.int64, device="cuda")
    stor = codec.store(xg, float(storage.noa_scale(1e-5, rng)))
    req, dst = 1e-2, 1e-4
    ea, eb = float(storage.noa_scale(req, rng)), float(storage.noa_scale(dst, rng))
    init, init_h = (torch.empty(cap, dtype=torch.uint8, device="cuda") for _ in range(2))
    cl, cl_h = torch.full_like(xg, 7.0), torch.full_like(xg, -7.0)
    codec.s2c_encode_apply_noa(stor, init, sz[0:1], mm, req, n, cl)
    codec.s2c_encode_apply(stor, init_h, sz[1:2], ea, n, cl_h)
    codec.sync()
    assert int(sz[0]) == int(sz[1]) and u8(init[: int(sz[0])]) == u8(init_h[: int(sz[1])])
    assert torch.equal(cl.view(torch.int32), cl_h.view(torch.int32))
    assert torch.equal(cl.view(torch.int32), codec.init_recv(init[: int(sz[0])]).view(torch.int32))
    before = cl.clone()
    resi, resi_h = (torch.empty(cap, dtype=torch.uint8, device="cuda") for _ in range(2))
    codec.residual_encode_apply_noa(stor, resi, sz[2:3], mm, req, dst, n, cl)
    codec.residual_encode_apply(stor, resi_h, sz[3:4], ea, eb, n, cl_h)
    codec.sync()
    assert int(sz[2]) == int(sz[3]) and u8(resi[: int(sz[2])]) == u8(resi_h[: int(sz[3])])
    assert u8(resi[: int(sz[2])]) == O.resi_send(u8(stor), ea, eb)
    assert torch.equal(cl.view(torch.int32), cl_h.view(torch.int32))
    assert torch.equal(cl.view(torch.int32), codec.resi_recv(before, resi[: int(sz[2])]).view(torch.int32))


def test_device_noa_bound_errors_are_latched(codec):
    from cortado_b200._native import CortadoError
    from cortado_b200.ops import max_stream_bytes
    x = torch.full((8192,), 3.0, device="cuda")  # range 0: every NOA bound is 0
    mm = codec.INOA_find_range_device(x)
    out = torch.full((max_stream_bytes(x.numel() * 4),), 0x5A, dtype=torch.uint8, device="cuda")
    sz = torch.full((1,), -7, dtype=torch.int64, device="cuda")
    for eb, want in ((1e-3, "EB_TOO_SMALL"),):
        codec.server_encode_noa(x, x.numel() * 4, out, sz, mm, eb)
        with pytest.raises(CortadoError) as e:
            codec.sync()
        assert e.value.name == want
        assert int(sz.item()) == -7 and bool((out == 0x5A).all())  # nothing written
    y = fields.mixed_field(8192, "white", 9).cuda()
    mm = codec.INOA_find_range_device(y)
    codec.server_encode_noa(y, y.numel() * 4, out, sz, mm, 3e38)  # bound exponent beyond the float range
    with pytest.raises(CortadoError) as e:
        codec.sync()
    assert e.value.name == "EB_TOO_LARGE"
    # the fused forms latch the same error and write neither the stream nor the client
    cl = torch.full_like(y, 5.0)
    stor = codec.store(y, 1e-3)
    codec.s2c_encode_apply_noa(stor, out, sz, mm, 3e38, y.numel() * 4, cl)
    with pytest.raises(CortadoError) as e:
        codec.sync()
    assert e.value.name == "EB_TOO_LARGE"
    assert int(sz.item()) == -7 and bool((out == 0x5A).all()) and bool((cl == 5.0).all())
    codec.server_encode_noa(y, y.numel() * 4, out, sz, mm, 1e-3)  # the context stays usable
    codec.sync()
    assert int(sz.item()) > 0


def test_noa_flow_captured_in_a_graph(codec, cuda_device):
    from cortado_b200.ops import max_stream_bytes
    x = fields.sinusoid((64, 128, 128), 2, outlier_frac=1e-3, device=cuda_device).reshape(-1)
    n = x.numel() * 4
    cap = max_stream_bytes(n)
    mm = torch.empty(2, dtype=torch.float32, device=cuda_device)
    stor, init, resi = (torch.empty(cap, dtype=torch.uint8, device=cuda_device) for _ in range(3))
    cl, fin = torch.empty_like(x), torch.empty_like(x)
    sz = torch.zeros(5, dtype=torch.int64, device=cuda_device)
    s = torch.cuda.Stream(cuda_device)

    def flow():
        codec.INOA_find_range_device(x, mm, stream=s)
        codec.server_encode_noa(x, n, stor, sz[0:1], mm, 1e-4, stream=s)
        codec.s2c_encode_noa(stor, init, sz[1:2], mm, 1e-2, n, stream=s)
        codec.client_decode(init, cl, sz[2:3], stream=s)
        codec.residual_encode_noa(stor, resi, sz[3:4], mm, 1e-2, 1e-4, n, stream=s)
        codec.residual_apply(cl, n, resi, fin, sz[4:5], stream=s)

    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        flow()  # eager once: the context's scratch is sized before capture
    codec.sync(s)
    eager = [stor[: int(sz[0])].clone(), init[: int(sz[1])].clone(), resi[: int(sz[3])].clone(), fin.clone()]
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        flow()
    for t in (stor, init, resi):
        t.fill_(0)
    fin.zero_()
    g.replay()
    torch.cuda.synchronize()
    codec.sync(s)
    assert torch.equal(stor[: int(sz[0])], eager[0]) and torch.equal(init[: int(sz[1])], eager[1])
    assert torch.equal(resi[: int(sz[3])], eager[2]) and torch.equal(fin.view(torch.int32), eager[3].view(torch.int32))
    xn = x.cpu().numpy()
    rng = O.noa_range(xn)
    eb = float(storage.noa_scale(1e-4, rng))
    assert np.array_equal(fin.cpu().numpy().view(np.uint32), O.client_roundtrip(xn, eb).view(np.uint32))
    del g
