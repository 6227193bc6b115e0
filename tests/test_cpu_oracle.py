"""CPU tests of the oracle itself: its BIT_4 emulation equals the closed-form
MSB-first bit transpose, RZE_1 round-trips and fails exactly where the
reference's capacity checks fail, the quantizers keep their bounds, and the
nested-bin identity the reference's -v paths check holds."""
import numpy as np
import pytest

from oracle import oracle as O


def closed_form_bit4(words: np.ndarray) -> np.ndarray:
    """Plane s of a 32-word group holds bit (31-s) of word i at bit (31-i)."""
    out = np.zeros(32, np.uint32)
    for s in range(32):
        col = (words >> np.uint32(31 - s)) & np.uint32(1)
        out[s] = np.uint32(sum(int(col[i]) << (31 - i) for i in range(32)))
    return out


@pytest.mark.parametrize("seed", range(4))
def test_bit4_is_msb_first_transpose(seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    w = rng.integers(0, 2**32, 4096, dtype=np.uint64).astype(np.uint32)
    out = O.bit4(w.view(np.uint8)).view(np.uint32)
    G = 128
    for g in (0, 5, 127):
        planes = closed_form_bit4(w[32 * g: 32 * g + 32])
        assert np.array_equal(out[g + G * np.arange(32)], planes)
    assert np.array_equal(O.ibit4(out.view(np.uint8)).view(np.uint32), w)


@pytest.mark.parametrize("nbytes", [4, 100, 124, 128, 132, 3232, 16380, 16384])
def test_bit4_partial_chunk_roundtrip(nbytes):
    rng = np.random.Generator(np.random.PCG64(nbytes))
    b = rng.integers(0, 256, nbytes, dtype=np.uint8)
    t = O.bit4(b)
    extra = nbytes % 128
    assert np.array_equal(t[nbytes - extra:], b[nbytes - extra:])
    assert np.array_equal(O.ibit4(t), b)


def test_rze_roundtrip_and_layout():
    rng = np.random.Generator(np.random.PCG64(1))
    for density in (0.0, 0.01, 0.2, 0.6):
        b = (rng.random(16384) < density) * rng.integers(1, 256, 16384)
        b = b.astype(np.uint8)
        enc = O.rze(b)
        if density == 0.0:
            assert enc is not None and enc.tolist() == [0x00, 0x40]  # trailer only: csize 16384
            continue
        if enc is None:
            continue
        assert int(enc[-2]) | (int(enc[-1]) << 8) == 16384
        nz = b[b != 0]
        assert np.array_equal(enc[: nz.size], nz)  # zero-eliminated bytes lead the payload
        assert np.array_equal(O.irze(enc), b)


def test_rze_rejects_incompressible():
    rng = np.random.Generator(np.random.PCG64(2))
    b = rng.integers(1, 256, 16384, dtype=np.uint8)
    assert O.rze(b) is None


def test_rze_capacity_boundary():
    # non-zero byte count just below / at the ZE limit (avail = CS - 2)
    b = np.zeros(16384, np.uint8)
    b[:16381] = 7
    enc = O.rze(b)
    assert enc is None or len(enc) >= 16381
    b[:16382] = 7
    assert O.rze(b) is None


@pytest.mark.parametrize("eb", [1e-1, 3e-3, 1e-5, 1e-30])
def test_quantizer_bounds(eb):
    rng = np.random.Generator(np.random.PCG64(3))
    x = np.concatenate([rng.standard_normal(20000).astype(np.float32),
                        (rng.standard_normal(1000) * 1e6).astype(np.float32),
                        np.array([0.0, -0.0, 1e-40, -1e-38, 3.4e38], np.float32)])
    rt = O.client_roundtrip(x, eb)
    assert O.maxabs(rt, x, eb) == -1
    e, t, o = O.eb_params(eb / 2)
    xs = x.view(np.uint32)
    for i in range(0, x.size, 97):
        d = O.iq(O.sq(int(xs[i]), e), e)
        assert abs(float(np.uint32(d).view(np.float32)) - float(x[i])) <= eb


def test_nested_bins_identity():
    """iCQ(CQ(iSQ(SQ(x, eb_s/2)), eb_c)) == iCQ(CQ(x, eb_c)) whenever eb_c >= eb_s
    (the property the reference's init_bench -v checks bit for bit)."""
    rng = np.random.Generator(np.random.PCG64(4))
    x = (rng.standard_normal(50000) * 3).astype(np.float32)
    for eb_s, eb_c in ((1e-5, 1e-2), (1e-4, 1e-4), (2e-3, 5e-3)):
        stor = O.store_encode(x, eb_s)
        init = O.init_send(stor, eb_c)
        assert np.array_equal(O.init_recv(init).view(np.uint32), O.client_roundtrip(x, eb_c).view(np.uint32))


def test_eb_errors():
    with pytest.raises(O.OracleError) as e:
        O.store_encode(np.ones(10, np.float32), 1e-39)
    assert e.value.code == 1
    with pytest.raises(O.OracleError) as e:
        O.store_encode(np.ones(10, np.float32), 3e38)
    assert e.value.code == 2


def test_corrupt_streams_detected():
    x = np.sin(np.arange(40000, dtype=np.float32) / 100)
    s = bytearray(O.store_encode(x, 1e-3))
    with pytest.raises(O.OracleError):
        O.store_decode(bytes(s[:20]))
    bad = bytearray(s)
    bad[16] = 0xFF
    bad[17] = 0xFF  # chunk 0 size 65535 > 16384
    with pytest.raises(O.OracleError):
        O.store_decode(bytes(bad))
