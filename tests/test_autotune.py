"""Autotuner: CPU tests of its cache and size classes; on the GPU, the launch
shape it sets changes no output byte."""
import json

import pytest
import torch

from cortado_b200 import autotune


def test_size_classes_and_cache_roundtrip(tmp_path, monkeypatch):
    monkeypatch.setenv("CORTADO_TUNE_CACHE", str(tmp_path / "t.json"))
    assert autotune.size_class(1 << 20) == "le4MiB"
    assert autotune.size_class(100 << 20) == "le512MiB"
    assert autotune.size_class(2 << 30) == "gt512MiB"
    assert autotune.load_cache() == {}
    autotune.save_cache({"k": {"store": {"ctas_per_sm": 4}}})
    assert json.load(open(tmp_path / "t.json"))["k"]["store"]["ctas_per_sm"] == 4


@pytest.mark.gpu
def test_launch_shape_never_changes_bytes(cuda_device, tmp_path, monkeypatch):
    from cortado_b200 import fields
    from cortado_b200.ops import Codec
    monkeypatch.setenv("CORTADO_TUNE_CACHE", str(tmp_path / "t.json"))
    c = Codec(cuda_device.index)
    best = autotune.tune(c, n_bytes=8 << 20, candidates=(1, 3, 6), reps=2)
    assert set(best) == set(autotune.OPS)
    x = fields.mixed_field(3 * 1024 * 1024 // 4 + 77, "grf", 3).to(cuda_device)
    ref = c.store(x, 1e-3)
    for k in (1, 2, 5, 0):
        c.set_launch_ctas("store", k)
        assert torch.equal(c.store(x, 1e-3), ref)
    c.close()
