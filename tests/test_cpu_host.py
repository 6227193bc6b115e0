"""CPU tests of the host-side logic (bounds, storage files, request planning)
and of the C-ABI library's load and exports (no compute calls without a GPU)."""
import ctypes
import os
import re

import numpy as np

from cortado_b200 import storage

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_store_bounds_sorted_deduped_scaled():
    user, absb = storage.store_bounds(["1e-5", "1e-1", "1e-3", "1e-1"], False, np.float32(2.5))
    assert user == [np.float32(1e-1), np.float32(1e-3), np.float32(1e-5)]
    assert absb == [np.float32(np.float32(2.5) * np.float32(e)) for e in user]
    user, absb = storage.store_bounds([1e-2, 1e-4], True, np.float32(7.0))
    assert absb == user


def test_select_stored_first_not_above():
    ebs = [np.float32(1e-1), np.float32(1e-3), np.float32(1e-5)]
    assert storage.select_stored(ebs, 1e-2) == 1
    assert storage.select_stored(ebs, 1e-1) == 0
    assert storage.select_stored(ebs, 1e-5) == 2
    assert storage.select_stored(ebs, 1e-6) == -1


def test_meta_roundtrip_layout(tmp_path):
    m = storage.StorMeta("data/x.f32", [np.float32(0.2), np.float32(0.002)], np.float32(2.0))
    b = storage.pack_meta(m)
    # int32 name_len, int32 n, float ebs[n], float range, name (util.h:70-99)
    assert b[:8] == bytes([10, 0, 0, 0, 2, 0, 0, 0])
    assert b[-10:] == b"data/x.f32"
    m2 = storage.unpack_meta(b)
    assert m2.name == m.name and m2.ebs == m.ebs and m2.range == m.range
    storage.write_storage(str(tmp_path / "st"), "data/x.f32", [b"a", b"bc"], m.ebs, m.range)
    assert sorted(os.listdir(tmp_path / "st")) == [".stor.meta", "x.f32.stor.00", "x.f32.stor.01"]
    assert storage.read_storage_meta(str(tmp_path / "st")).ebs == m.ebs


def test_plans():
    rng = np.float32(10.0)
    _, ebs = storage.store_bounds(["1e-2", "1e-4"], False, rng)
    meta = storage.StorMeta("x", ebs, rng)
    p = storage.plan_init(meta, "1e-2", abs_mode=False)
    assert p.stored_index == 0 and p.eb1_abs == np.float32(rng * np.float32(1e-2))
    # float32(10) * float32(0.01) rounds below float32(0.1): the coarser file does not qualify
    meta = storage.StorMeta("x", [np.float32(0.1), np.float32(0.001)], rng)
    assert storage.plan_init(meta, "1e-2", abs_mode=False).stored_index == 1
    assert storage.plan_resi(meta, "1e-2", "1e-4", abs_mode=False).stored_index == -1  # too tight
    _, ebs = storage.store_bounds(["1e-1", "1e-4"], False, rng)
    p = storage.plan_resi(storage.StorMeta("x", ebs, rng), "1e-2", "1e-4", abs_mode=False)
    assert p.stored_index == 1


def test_max_stream_bytes():
    assert storage.max_stream_bytes(0) == 16
    assert storage.max_stream_bytes(4) == 16 + 2 + 16384
    assert storage.max_stream_bytes(16384 * 3) == 16 + 6 + 3 * 16384


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "cortado.h")).read()
    return sorted(set(re.findall(r"\b(cortado_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from cortado_b200 import build
    lib_path = build.build()
    L = ctypes.CDLL(lib_path)
    syms = _declared_symbols()
    assert len(syms) >= 12
    for s in syms:
        assert hasattr(L, s), s
    from cortado_b200 import _native
    assert set(_native.SIGNATURES) == set(syms)


def test_host_only_entry_points_without_gpu():
    from cortado_b200 import _native
    L = _native.lib()
    assert L.cortado_max_stream_bytes(16384) == 16 + 2 + 16384
    e = ctypes.c_int()
    assert L.cortado_eb_exponent(ctypes.c_float(1.0), ctypes.byref(e)) == 0 and e.value == 127
    assert L.cortado_eb_exponent(ctypes.c_float(1e-39), ctypes.byref(e)) == 1
    assert L.cortado_eb_exponent(ctypes.c_float(1e37), ctypes.byref(e)) == 2
    assert L.cortado_status_string(3) == b"corrupt stream"
