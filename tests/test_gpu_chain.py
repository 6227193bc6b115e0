"""The progressive chain captured as a CUDA graph: every replay reproduces the
eager run's streams and reconstructions bit for bit, every reconstruction
satisfies its bound on the device, and each step equals iCQ(CQ(x)) at its
bound (the identity the reference's resi_bench -v checks)."""
import numpy as np
import pytest
import torch

from cortado_b200 import fields, storage
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_chain_graph_matches_eager_and_bounds(cuda_device):
    from cortado_b200.chain import ProgressiveChain
    from cortado_b200.ops import Codec
    codec = Codec(cuda_device.index)
    x = fields.grf((1024, 1024), 4, slope=2.5, device=cuda_device).reshape(-1)
    lo, hi = codec.INOA_find_range(x)
    rng = storage.value_range(lo, hi)
    nb = lambda e: float(storage.noa_scale(e, rng))
    ch = ProgressiveChain(codec, x, [nb(1e-1), nb(1e-3), nb(1e-5), nb(1e-7)], nb(1e-1),
                          [nb(1e-2), nb(1e-3), nb(1e-4), nb(1e-5), nb(1e-6)])
    ch.run_eager()
    codec.sync()
    eager = [r.clone() for r in ch.recon]
    eager_streams = [s[: int(n)].clone() for s, n in zip(ch.streams, ch.stream_sizes.tolist())]
    assert (ch.first_bad == -1).all()
    xn = x.cpu().numpy()
    for r, eb in zip(eager, ch.bounds):
        assert np.array_equal(r.cpu().numpy().view(np.uint32), O.client_roundtrip(xn, eb).view(np.uint32))
    ch.capture()
    for _ in range(2):
        for r in ch.recon:
            r.zero_()
        ch.first_bad.fill_(7)
        ch.replay()
        torch.cuda.synchronize()
        codec.sync()
        assert (ch.first_bad == -1).all()
        for a, b in zip(eager, ch.recon):
            assert torch.equal(a.view(torch.int32), b.view(torch.int32))
        for a, s, n in zip(eager_streams, ch.streams, ch.stream_sizes.tolist()):
            assert torch.equal(a, s[: int(n)])
    codec.close()


def test_verify_bound_matches_oracle(cuda_device):
    from cortado_b200.ops import Codec
    codec = Codec(cuda_device.index)
    rng = np.random.Generator(np.random.PCG64(5))
    x = rng.standard_normal(100000).astype(np.float32)
    x[:5] = [np.nan, np.inf, -np.inf, 0.0, -0.0]
    for eb in (1e-3, 1e-1):
        r = x + rng.uniform(-eb, eb, x.size).astype(np.float32)
        r[:5] = x[:5]
        for bad_at in (None, 77777, 3):
            rr = r.copy()
            if bad_at is not None:
                rr[bad_at] = rr[bad_at] + 10 * eb if bad_at != 3 else np.float32(1.0)  # 3: 0.0 -> 1.0
            got = int(codec.verify_bound(torch.from_numpy(x).cuda(), torch.from_numpy(rr).cuda(), eb).item())
            assert got == O.maxabs(rr, x, eb)
    codec.close()
