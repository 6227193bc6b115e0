"""cortado_store_encode_noalloc: the store entry point for callers that cannot
allocate device memory (for example code inside a framework that owns the
device's whole memory pool, or a real-time path that must not hit an
allocation's implicit synchronization).  It uses a fixed scratch array built
into the library instead of a context.  This file is collected last so that a
failure here does not hide the other tests' results; it must pass both on its
own in a fresh process and after the rest of the suite."""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def _call_noalloc(L, x, eb, out, size):
    st = torch.cuda.current_stream().cuda_stream
    return L.cortado_store_encode_noalloc(x.data_ptr(), x.numel() * 4, ctypes.c_float(eb), out.data_ptr(),
                                          out.numel(), size.data_ptr(), st)


def test_noalloc_matches_context_store_twice(cuda_device):
    from cortado_b200 import _native, fields
    from cortado_b200.ops import Codec, max_stream_bytes
    L = _native.lib()
    # one full-size chunk run plus a partial last chunk; errors in both paths show
    x = fields.sinusoid((64, 64, 65), 21).reshape(-1).to(cuda_device)
    eb = 1e-3
    codec = Codec(cuda_device.index)
    expected = codec.store(x, eb)  # the existing, context-based entry point
    codec.close()
    cap = max_stream_bytes(x.numel() * 4)
    for _ in range(2):  # the shared scratch keeps the previous call's contents
        out = torch.full((cap,), 0xAB, dtype=torch.uint8, device=cuda_device)
        size = torch.zeros(1, dtype=torch.int64, device=cuda_device)
        assert _call_noalloc(L, x, eb, out, size) == 0
        torch.cuda.synchronize()
        n = int(size.item())
        assert n == expected.numel()
        assert torch.equal(out[:n], expected)  # integer codec: exact equality


def test_noalloc_rejects_inputs_beyond_scratch(cuda_device):
    from cortado_b200 import _native
    L = _native.lib()
    x = torch.empty(4, dtype=torch.float32, device=cuda_device)
    out = torch.empty(64, dtype=torch.uint8, device=cuda_device)
    size = torch.zeros(1, dtype=torch.int64, device=cuda_device)
    too_big = (1 << 30) + 4
    st = torch.cuda.current_stream().cuda_stream
    rc = L.cortado_store_encode_noalloc(x.data_ptr(), too_big, ctypes.c_float(1e-3), out.data_ptr(), 1 << 40,
                                        size.data_ptr(), st)
    assert _native.STATUS_NAMES[rc] == "SCRATCH_LIMIT"


def test_noalloc_epoch_wrap_and_largest_input(cuda_device):
    """Two further cases on the one shared scratch: (1) a store 65,536 calls
    after another runs at the same 16-bit epoch, which only the clear at the
    epoch's wrap keeps from reading the older call's lookback words; (2) an
    input of exactly CORTADO_NOALLOC_MAX_BYTES (1 GiB), compared with the
    oracle directly."""
    from cortado_b200 import _native, fields
    from cortado_b200.ops import max_stream_bytes
    from oracle import oracle as O
    L = _native.lib()
    eb = 1e-3
    xa = fields.mixed_field(100 * 4096 + 57, "sinusoid", 41).to(cuda_device)
    xb = fields.mixed_field(100 * 4096 + 57, "white", 42).to(cuda_device)
    cap = max_stream_bytes(xa.numel() * 4)
    oa, ob = (torch.empty(cap, dtype=torch.uint8, device=cuda_device) for _ in range(2))
    sa, sb = (torch.zeros(1, dtype=torch.int64, device=cuda_device) for _ in range(2))
    tiny = fields.white(4096, 6).to(cuda_device)
    tout = torch.empty(max_stream_bytes(tiny.numel() * 4), dtype=torch.uint8, device=cuda_device)
    tsz = torch.zeros(1, dtype=torch.int64, device=cuda_device)
    assert _call_noalloc(L, xa, eb, oa, sa) == 0
    for _ in range(65535):  # one of these calls has epoch 65535 and clears the words
        assert _call_noalloc(L, tiny, eb, tout, tsz) == 0
    assert _call_noalloc(L, xb, eb, ob, sb) == 0  # the same epoch as xa's call
    torch.cuda.synchronize()
    assert bytes(ob[: int(sb.item())].cpu().numpy()) == O.store_encode(xb.cpu().numpy(), eb)
    assert bytes(oa[: int(sa.item())].cpu().numpy()) == O.store_encode(xa.cpu().numpy(), eb)
    del xa, xb, oa, ob
    n = 1 << 30  # CORTADO_NOALLOC_MAX_BYTES
    x = fields.grf((16384, 16384), 9, slope=2.5, device=cuda_device).reshape(-1)
    assert x.numel() * 4 == n
    out = torch.empty(max_stream_bytes(n), dtype=torch.uint8, device=cuda_device)
    size = torch.zeros(1, dtype=torch.int64, device=cuda_device)
    ebx = 1e-4
    assert _call_noalloc(L, x, ebx, out, size) == 0
    torch.cuda.synchronize()
    got = bytes(out[: int(size.item())].cpu().numpy())
    del out
    assert got == O.store_encode(x.cpu().numpy(), ebx)
