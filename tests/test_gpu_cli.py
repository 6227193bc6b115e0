"""The command-line drivers, run with the reference CLIs' arguments, write the
same files the reference's binaries wrote (tests/golden/reference_outputs.json):
the drop-in test for the file formats and the bound plumbing."""
import hashlib
import os
import subprocess

import numpy as np
import pytest

from cortado_b200 import build
from tests import golden_cases as G

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(build.LIB), "bin")


def _run(args, cwd):
    r = subprocess.run(args, cwd=cwd, capture_output=True, text=True, timeout=300)
    return r.returncode, r.stdout + r.stderr


@pytest.mark.parametrize("name,setting", [c for c in G.cases() if c[0] in
                                          ("sin3d_32", "sin1d_partial", "noise_64k", "randbits", "one_chunk_plus1")],
                         ids=lambda v: v if isinstance(v, str) else v["tag"])
def test_cli_files_match_reference(cuda_device, tmp_path, name, setting):
    build.build()
    ref = G.reference_outputs().get(f"{name}/{setting['tag']}")
    if ref is None:
        pytest.skip("no reference record")
    src = os.path.join(G.GOLDEN, "inputs", name + ".f32")
    inp = tmp_path / (name + ".f32")
    inp.write_bytes(open(src, "rb").read())
    flag = ["-a"] if setting["mode"] == "abs" else []
    rc, out = _run([os.path.join(BIN, "store"), str(inp), *setting["store"], *flag, "-o", "stor"], tmp_path)
    assert rc == 0, out
    for idx, rec in ref["stor"].items():
        b = (tmp_path / "stor" / f"{name}.f32.stor.{idx}").read_bytes()
        assert {"sha256": G.stream_hash(b), "bytes": len(b)} == rec, idx
    meta = (tmp_path / "stor" / ".stor.meta").read_bytes()
    n = int.from_bytes(meta[4:8], "little")
    ebs = list(np.frombuffer(meta, np.uint32, n, 8))
    assert ebs == ref["meta"]["ebs"]
    assert int(np.frombuffer(meta, np.uint32, 1, 8 + 4 * n)[0]) == ref["meta"]["range"]
    rc, out = _run([os.path.join(BIN, "init_send"), "stor", setting["init"], *flag, "-c", "init.bin"], tmp_path)
    assert rc == 0, out
    b = (tmp_path / "init.bin").read_bytes()
    assert {"sha256": G.stream_hash(b), "bytes": len(b)} == ref["init.bin"]
    rc, out = _run([os.path.join(BIN, "init_recv"), "init.bin", "-d", "init_dec.f32"], tmp_path)
    assert rc == 0, out
    b = (tmp_path / "init_dec.f32").read_bytes()
    assert {"sha256": hashlib.sha256(b).hexdigest(), "bytes": len(b)} == ref["init_dec.f32"]
    rc, out = _run([os.path.join(BIN, "resi_send"), "stor", *setting["resi"], *flag, "-c", "resi.bin"], tmp_path)
    assert rc == 0, out
    b = (tmp_path / "resi.bin").read_bytes()
    assert {"sha256": G.stream_hash(b), "bytes": len(b)} == ref["resi.bin"]
    rc, out = _run([os.path.join(BIN, "resi_recv"), "init_dec.f32", "resi.bin", "-d", "resi_dec.f32"], tmp_path)
    assert rc == 0, out
    if ref.get("resi_recv_deterministic", True):
        b = (tmp_path / "resi_dec.f32").read_bytes()
        assert {"sha256": hashlib.sha256(b).hexdigest(), "bytes": len(b)} == ref["resi_dec.f32"]


def test_store_replaces_output_dir_without_a_shell(cuda_device, tmp_path):
    """store -o deletes the output directory (with old contents, nested
    directories included) and creates it again, as the reference's
    std::filesystem calls do; no character of the path is interpreted (a
    quote, a space, a semicolon and a $ stay part of the name)."""
    build.build()
    src = os.path.join(G.GOLDEN, "inputs", "sin3d_32.f32")
    inp = tmp_path / "in.f32"
    inp.write_bytes(open(src, "rb").read())
    odd = "out dir 'q'; touch pwned; $HOME"
    d = tmp_path / "a" / odd
    (d / "old" / "deeper").mkdir(parents=True)
    (d / "old" / "deeper" / "stale.bin").write_bytes(b"x")
    (d / "stale.stor.07").write_bytes(b"y")
    rc, out = _run([os.path.join(BIN, "store"), str(inp), "1e-2", "1e-4", "-o", str(d)], tmp_path)
    assert rc == 0, out
    assert sorted(os.listdir(d)) == [".stor.meta", "in.f32.stor.00", "in.f32.stor.01"]
    assert not (tmp_path / "pwned").exists()
