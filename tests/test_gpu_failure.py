"""Failure detection without a GPU fault: a bounded device wait on a word that
nothing publishes gives up after the context's timeout, the host reads the
TIMEOUT status from sync(), the status is cleared, and the same context then
encodes and decodes correctly."""
import numpy as np
import pytest

from cortado_b200 import fields
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_recovers(cuda_device):
    from cortado_b200._native import CortadoError
    from cortado_b200.ops import Codec
    c = Codec(cuda_device.index)
    c.set_timeout(0.002)
    for _ in range(2):  # the latch is cleared by each report
        c.selftest_timeout()
        with pytest.raises(CortadoError) as e:
            c.sync()
        assert e.value.name == "TIMEOUT"
    c.sync()  # nothing latched any more
    c.set_timeout(2.0)
    x = fields.sinusoid((32, 64, 64), 3).reshape(-1)
    s = c.store(x.to(cuda_device), 1e-3)
    assert bytes(s.cpu().numpy()) == O.store_encode(x.numpy(), 1e-3)
    d = c.store_decode(s)
    assert np.array_equal(d.cpu().numpy().view(np.uint32), O.store_decode(O.store_encode(x.numpy(), 1e-3)).view(np.uint32))
    c.close()
