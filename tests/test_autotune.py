"""Autotuner: CPU tests of its cache, size classes, lookup order and choice
rule; on the GPU, a tuning run picks parameters for every operation, a cache
hit applies them to a new context (launch shape and resolver change), and no
setting changes an output byte."""
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


def test_lookup_prefers_cache_then_shipped_table(tmp_path, monkeypatch):
    monkeypatch.setenv("CORTADO_TUNE_CACHE", str(tmp_path / "t.json"))
    monkeypatch.setattr(autotune, "gpu_name", lambda device: "Test GPU")
    monkeypatch.setattr(autotune, "shipped_path", lambda device: str(tmp_path / "Test_GPU.json"))
    assert autotune.lookup(0, 1 << 28) == (None, "defaults")
    (tmp_path / "Test_GPU.json").write_text(json.dumps({"le512MiB": {"store": {"ctas_per_sm": 5, "resolver": 1}}}))
    assert autotune.lookup(0, 1 << 28) == ({"store": {"ctas_per_sm": 5, "resolver": 1}}, "shipped")
    assert autotune.lookup(0, 1 << 20) == (None, "defaults")
    autotune.save_cache({"Test GPU|le512MiB": {"store": {"ctas_per_sm": 3, "resolver": 0}}})
    assert autotune.lookup(0, 1 << 28) == ({"store": {"ctas_per_sm": 3, "resolver": 0}}, "cache")


def test_choice_treats_near_ties_as_equal_and_prefers_occupancy():
    # 5 CTAs per SM faster by 0.2%: a tie, 6 wins
    assert autotune.choose({(5, 1): 0.3094, (6, 1): 0.3101, (6, 0): 0.3107, (3, 1): 0.39}) == (6, 1)
    assert autotune.choose({(5, 1): 0.3046, (6, 1): 0.3078, (6, 0): 0.3108}) == (6, 1)
    # faster by more than the tie: kept
    assert autotune.choose({(5, 1): 0.300, (6, 1): 0.320}) == (5, 1)
    # resolver on and off tied at the same CTAs: on
    assert autotune.choose({(6, 0): 0.3100, (6, 1): 0.3102}) == (6, 1)
    assert autotune.choose({(4, 1): 1.0}) == (4, 1)


@pytest.mark.gpu
def test_tuned_parameters_never_change_bytes(cuda_device, tmp_path, monkeypatch):
    from cortado_b200 import fields
    from cortado_b200.ops import Codec
    monkeypatch.setenv("CORTADO_TUNE_CACHE", str(tmp_path / "t.json"))
    c = Codec(cuda_device.index, tuned=False)
    best = autotune.tune(c, n_bytes=8 << 20, ctas=(1, 3, 6), reps=2)
    assert set(best) == set(autotune.OPS)
    assert all(v["ctas_per_sm"] in (1, 3, 6) for v in best.values())
    autotune.save_cache({autotune.key(cuda_device, 256 << 20): best})
    c2 = Codec(cuda_device.index)  # picks the cached table up
    assert c2.tuning["source"] == "cache" and c2.tuning["params"] == best
    x = fields.mixed_field(3 * 1024 * 1024 // 4 + 77, "grf", 3).to(cuda_device)
    ref = c.store(x, 1e-3)
    ref_init = c.init_send(ref, 1e-2)
    ref_resi = c.resi_send(ref, 1e-2, 1e-3)
    for k, res in ((1, 0), (2, 1), (5, 0), (0, 1)):
        for op in ("store", "init_send", "resi_send"):
            c2.set_launch_ctas(op, k)
            c2.set_resolver(op, bool(res))
        s = c2.store(x, 1e-3)
        assert torch.equal(s, ref)
        assert torch.equal(c2.init_send(s, 1e-2), ref_init)
        assert torch.equal(c2.resi_send(s, 1e-2, 1e-3), ref_resi)
    c.close()
    c2.close()
