"""The 16-bit launch epoch of a context wraps after 65,536 launches.  Lookback
and payload-offset words are tagged with the epoch of the launch that wrote
them, so at the wrap (the launch with epoch 65535) the last CTA clears them
all; otherwise a launch 65,536 launches later, at the same epoch, would read
an old launch's words as its own.  Here a multi-chunk store and decode run,
then 65,534 one-chunk launches, then a store and a decode of other data at
exactly the same epochs as the first two: their outputs must equal the
oracle's."""
import numpy as np
import pytest
import torch

from cortado_b200 import fields
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EPOCHS = 65536


def test_context_epoch_wrap_clears_old_words(cuda_device):
    from cortado_b200.ops import Codec, max_stream_bytes
    eb = 1e-3
    xa = fields.mixed_field(100 * 4096 + 123, "sinusoid", 31).to(cuda_device)
    xb = fields.mixed_field(100 * 4096 + 123, "grf", 32).to(cuda_device)
    prep = Codec(cuda_device.index)  # streams made on another context leave this one's epoch alone
    init_a = prep.init_send(prep.store(xa, eb), eb * 10)
    init_b = prep.init_send(prep.store(xb, eb), eb * 10)
    prep.close()
    c = Codec(cuda_device.index)  # fresh context: epoch 0
    n = xa.numel() * 4
    cap = max_stream_bytes(n)
    sa, sb = (torch.empty(cap, dtype=torch.uint8, device=cuda_device) for _ in range(2))
    da, db = torch.empty_like(xa), torch.empty_like(xb)
    sz = torch.zeros(4, dtype=torch.int64, device=cuda_device)
    tiny = fields.white(4096, 5).to(cuda_device)
    tout = torch.empty(max_stream_bytes(tiny.numel() * 4), dtype=torch.uint8, device=cuda_device)
    tsz = torch.zeros(1, dtype=torch.int64, device=cuda_device)
    c.server_encode(xa, n, sa, sz[0:1], eb)              # epoch 0: lookback words of 101 chunks
    c.client_decode(init_a, da, sz[1:2])                 # epoch 1: payload offsets of 101 chunks
    for _ in range(EPOCHS - 2):                          # epochs 2 .. 65535 (the last one clears)
        c.server_encode(tiny, tiny.numel() * 4, tout, tsz, eb)
    c.server_encode(xb, n, sb, sz[2:3], eb)              # epoch 0 again
    c.client_decode(init_b, db, sz[3:4])                 # epoch 1 again
    c.sync()
    xbn = xb.cpu().numpy()
    stor_b = O.store_encode(xbn, eb)
    assert bytes(sb[: int(sz[2].item())].cpu().numpy()) == stor_b
    want = O.init_recv(O.init_send(stor_b, eb * 10))
    assert np.array_equal(db.cpu().numpy().view(np.uint32), want.view(np.uint32))
    assert bytes(sa[: int(sz[0].item())].cpu().numpy()) == O.store_encode(xa.cpu().numpy(), eb)
    c.close()
