"""Parity of the CUDA path (libcortado through its C ABI) with the CPU oracle:
streams must be byte-identical and decoded floats bit-identical, on the golden
cases, on edge-case sizes and generators, and at full benchmark sizes (where
size-independent properties are also checked against torch)."""
import numpy as np
import pytest
import torch

from cortado_b200 import fields, storage
from oracle import oracle as O
from tests import golden_cases as G

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


class GpuImpl:
    def __init__(self, codec):
        self.c = codec

    def noa_range(self, x):
        return self.c.INOA_find_range(torch.from_numpy(x).cuda())

    def store(self, x, eb):
        return u8(self.c.store(torch.from_numpy(x).cuda(), eb))

    def init_send(self, stored, n, eb):
        return u8(self.c.init_send(torch.frombuffer(bytearray(stored), dtype=torch.uint8).cuda(), eb, n))

    def init_recv(self, s):
        return self.c.init_recv(torch.frombuffer(bytearray(s), dtype=torch.uint8).cuda()).cpu().numpy()

    def resi_send(self, stored, n, src, dst):
        return u8(self.c.resi_send(torch.frombuffer(bytearray(stored), dtype=torch.uint8).cuda(), src, dst, n))

    def resi_recv(self, src, s):
        return self.c.resi_recv(torch.from_numpy(np.ascontiguousarray(src)).cuda(),
                                torch.frombuffer(bytearray(s), dtype=torch.uint8).cuda()).cpu().numpy()


class OracleImpl:
    def noa_range(self, x):
        return np.nanmin(x), np.nanmax(x)

    def store(self, x, eb):
        return O.store_encode(x, eb)

    def init_send(self, stored, n, eb):
        return O.init_send(stored, eb)

    def init_recv(self, s):
        return O.init_recv(s)

    def resi_send(self, stored, n, src, dst):
        return O.resi_send(stored, src, dst)

    def resi_recv(self, src, s):
        return O.resi_recv(src, s)


CASES = G.cases()


@pytest.mark.parametrize("name,setting", CASES, ids=[f"{n}-{s['tag']}" for n, s in CASES])
def test_golden_flow_matches_oracle(codec, name, setting):
    x = G.load_input(name)
    g = G.run_flow(GpuImpl(codec), x, setting)
    o = G.run_flow(OracleImpl(), x, setting)
    if "store_error" in o:
        assert "store_error" in g
        return
    for k in ("stor", "meta", "init.bin", "init_dec.f32", "resi.bin", "resi_dec.f32"):
        assert g[k] == o[k], k


@pytest.mark.parametrize("name,setting", CASES, ids=[f"{n}-{s['tag']}" for n, s in CASES])
def test_golden_flow_matches_reference(codec, name, setting):
    ref = G.reference_outputs().get(f"{name}/{setting['tag']}")
    if ref is None:
        pytest.skip("no reference record")
    x = G.load_input(name)
    rec = G.run_flow(GpuImpl(codec), x, setting)
    diffs = G.compare(rec, ref)
    assert not diffs, diffs


def _sizes():
    return [4, 8, 124, 128, 132, 4096, 16380, 16384, 16388, 16384 + 128, 3 * 16384 + 777 * 4, 7 * 16384, 40 * 16384 + 64]


@pytest.mark.parametrize("nbytes", _sizes())
@pytest.mark.parametrize("kind", ["sinusoid", "white", "grf", "randbits"])
def test_all_ops_match_oracle(codec, nbytes, kind):
    nw = nbytes // 4
    if kind == "randbits":
        rng = np.random.Generator(np.random.PCG64(nbytes))
        xb = rng.integers(0, 2**23, nw, dtype=np.uint32) | (rng.integers(90, 160, nw, dtype=np.uint32) << 23)
        x = xb.view(np.float32)
    else:
        x = fields.mixed_field(nw, kind, seed=nbytes % 1000 + 7).numpy()
    xg = torch.from_numpy(x).cuda()
    rng_ = O.noa_range(x)
    for eb_noa in (1e-1, 1e-3, 1e-6):
        eb = float(storage.noa_scale(eb_noa, rng_)) if rng_ > 0 else 1e-3
        stor_o = O.store_encode(x, eb)
        stor_g = codec.store(xg, eb)
        assert u8(stor_g) == stor_o, ("store", eb_noa)
        dec_g = codec.store_decode(stor_g)
        assert np.array_equal(bits(dec_g), bits(O.store_decode(stor_o))), ("store_decode", eb_noa)
        req = eb * 10
        init_o = O.init_send(stor_o, req)
        init_g = codec.init_send(stor_g, req)
        assert u8(init_g) == init_o, ("init_send", eb_noa)
        cl_o = O.init_recv(init_o)
        cl_g = codec.init_recv(init_g)
        assert np.array_equal(bits(cl_g), bits(cl_o)), ("init_recv", eb_noa)
        resi_o = O.resi_send(stor_o, req, eb * 2)
        resi_g = codec.resi_send(stor_g, req, eb * 2)
        assert u8(resi_g) == resi_o, ("resi_send", eb_noa)
        fin_o = O.resi_recv(cl_o, resi_o)
        fin_g = codec.resi_recv(cl_g, resi_g)
        assert np.array_equal(bits(fin_g), bits(fin_o)), ("resi_recv", eb_noa)


@pytest.mark.parametrize("req,dst", [(10.0, 2.0), (0.5, 0.25), (0.25, 0.1), (4.0, 1.0), (1.0, 4.0), (3.0, 0.3), (1.0, 1.0)])
def test_requant_bound_orders_match_oracle(codec, req, dst):
    """init_send / resi_send with request and destination bounds above, equal
    to and below the stored bound (multiples of it), on a field whose warps mix
    lossy words with lossless outliers and infinities: the encoders choose
    between the fast forms and the integer forms word by word."""
    rng = np.random.Generator(np.random.PCG64(17))
    nw = 8 * 4096 + 300
    x = rng.normal(0, 1, nw).astype(np.float32)
    idx = rng.choice(nw, nw // 500, replace=False)
    x[idx] = (rng.choice([-1.0, 1.0], idx.size) * rng.uniform(1e5, 1e7, idx.size)).astype(np.float32)
    x[idx[:2]] = [np.inf, -np.inf]
    eb = 1e-3
    stor_o = O.store_encode(x, eb)
    stor_g = codec.store(torch.from_numpy(x).cuda(), eb)
    assert u8(stor_g) == stor_o
    init_o = O.init_send(stor_o, eb * req)
    init_g = codec.init_send(stor_g, eb * req)
    assert u8(init_g) == init_o
    cl_o = O.init_recv(init_o)
    cl_g = codec.init_recv(init_g)
    assert np.array_equal(bits(cl_g), bits(cl_o))
    resi_o = O.resi_send(stor_o, eb * req, eb * dst)
    resi_g = codec.resi_send(stor_g, eb * req, eb * dst)
    assert u8(resi_g) == resi_o
    assert np.array_equal(bits(codec.resi_recv(cl_g, resi_g)), bits(O.resi_recv(cl_o, resi_o)))


def test_noa_range_matches(codec):
    for seed in range(3):
        x = fields.white(100003 * 4 // 4, seed).numpy() * (seed + 1)
        lo, hi = codec.INOA_find_range(torch.from_numpy(x).cuda())
        assert lo == x.min() and hi == x.max()


def _flow_props(codec, x_dev, eb_store, eb_init, eb_dst):
    """Size-independent properties of one progressive round trip."""
    stor = codec.store(x_dev, eb_store)
    dec = codec.store_decode(stor)
    assert torch.all((dec - x_dev).abs() <= eb_store)
    init = codec.init_send(stor, eb_init)
    cl = codec.init_recv(init)
    resi = codec.resi_send(stor, eb_init, eb_dst)
    fin = codec.resi_recv(cl, resi)
    # init_recv(init_send(store(x))) and resi_recv(...) equal the client quantizer roundtrip
    return stor, init, cl, resi, fin


@pytest.mark.parametrize("eb_noa", [1e-2, 1e-4])
def test_c1_config_matches_oracle(codec, eb_noa):
    """128^3 sinusoid field (8 MiB, 512 chunks): every op byte-exact."""
    x = fields.sinusoid((128, 128, 128), 1).reshape(-1)
    xn = x.numpy()
    rng_ = O.noa_range(xn)
    eb = float(storage.noa_scale(eb_noa, rng_))
    stor_o = O.store_encode(xn, eb)
    stor_g = codec.store(x.cuda(), eb)
    assert u8(stor_g) == stor_o
    init_o = O.init_send(stor_o, eb * 100)
    assert u8(codec.init_send(stor_g, eb * 100)) == init_o
    resi_o = O.resi_send(stor_o, eb * 100, eb)
    assert u8(codec.resi_send(stor_g, eb * 100, eb)) == resi_o


def test_large_field_properties_and_parity(codec):
    """512^3 field with outliers (the large-field configuration): bounds hold
    on device, init/residual decode equal iCQ(CQ(x)), and the streams equal
    the oracle's."""
    x = fields.sinusoid((512, 512, 512), 2, outlier_frac=1e-3, device="cuda").reshape(-1)
    lo, hi = codec.INOA_find_range(x)
    rng_ = storage.value_range(lo, hi)
    eb_s = float(storage.noa_scale(1e-5, rng_))
    eb_i = float(storage.noa_scale(1e-3, rng_))
    eb_d = float(storage.noa_scale(1e-5, rng_))
    stor, init, cl, resi, fin = _flow_props(codec, x, eb_s, eb_i, eb_d)
    xn = x.cpu().numpy()
    assert np.array_equal(bits(cl), bits(O.client_roundtrip(xn, eb_i)))
    assert np.array_equal(bits(fin), bits(O.client_roundtrip(xn, eb_d)))
    assert u8(stor) == O.store_encode(xn, eb_s)
    assert u8(init) == O.init_send(u8(stor), eb_i)
    assert u8(resi) == O.resi_send(u8(stor), eb_i, eb_d)


def test_repeat_is_deterministic(codec):
    x = fields.sinusoid((64, 64, 64), 9).reshape(-1).cuda()
    a = codec.store(x, 1e-3)
    for _ in range(3):
        assert torch.equal(codec.store(x, 1e-3), a)
