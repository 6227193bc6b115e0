"""Host <-> device pipelines: the two-slot scheduler never lets a slot's
buffers be overwritten while they are still being read (many items through a
pipeline whose work depends on every input byte), and StorePipeline's streams
are byte-identical to one-at-a-time Codec.store and to the oracle."""
import numpy as np
import pytest
import torch

from cortado_b200 import fields, storage
from oracle import oracle as O

pytestmark = pytest.mark.gpu


class _Slot:
    def __init__(self, dev, n):
        self.stream = torch.cuda.Stream(dev)
        self.x = torch.empty(n, dtype=torch.float32, device=dev)
        self.y = torch.empty(n, dtype=torch.float32, device=dev)


def test_pipeline_slot_reuse(cuda_device):
    from cortado_b200.pipeline import Pipeline
    n, items = 1 << 22, 9
    hosts = [torch.full((n,), float(i + 1)).pin_memory() for i in range(items)]
    outs = [torch.empty(n).pin_memory() for _ in range(items)]
    slots = [_Slot(cuda_device, n) for _ in range(2)]

    def load(i, sl, s):
        sl.x.copy_(hosts[i], non_blocking=True)

    def run(i, sl, s):
        for _ in range(8):  # long enough that a missing wait would show
            torch.mul(sl.x, 1.0, out=sl.y)
        sl.y.add_(sl.x)

    def store(i, sl, s):
        outs[i].copy_(sl.y, non_blocking=True)

    p = Pipeline(cuda_device, slots, load, run, store)
    p(items)
    p.sync()
    for i in range(items):
        assert torch.all(outs[i] == 2.0 * (i + 1)), i


def test_store_pipeline_matches_codec_and_oracle(cuda_device):
    from cortado_b200.ops import Codec
    from cortado_b200.pipeline import StorePipeline
    sizes = [4096 * 40 + 300, 4096 * 3, 77, 4096 * 17 + 1]
    kinds = ["sinusoid", "grf", "white", "sinusoid"]
    xs = [fields.mixed_field(n, k, 20 + i) for i, (n, k) in enumerate(zip(sizes, kinds))]
    bounds = []
    for x in xs:
        r = O.noa_range(x.numpy())
        bounds.append([float(storage.noa_scale(e, r)) for e in (1e-2, 1e-4)])
    sp = StorePipeline(cuda_device, max(sizes) * 4, 2)
    got = sp.run(xs, bounds)
    sp.close()
    c = Codec(cuda_device.index)
    for i, x in enumerate(xs):
        for j, eb in enumerate(bounds[i]):
            ref = c.store(x.to(cuda_device), eb).cpu()
            assert torch.equal(got[i][j], ref), (i, j)
    c.close()
    assert bytes(got[0][1].numpy()) == O.store_encode(xs[0].numpy(), bounds[0][1])
