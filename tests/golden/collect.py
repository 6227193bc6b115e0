"""Collects the outputs of tests/golden/run_reference.sh (reference binaries
run on a GPU box) into tests/golden/reference_outputs.json: per case and mode,
the sha256 and size of every stream (header bytes 12..15 zeroed -- the
reference leaves them unwritten), of every decoded file, the parsed
.stor.meta fields and the exit codes.

Usage: python tests/golden/collect.py <golden-output-dir>
"""
import hashlib
import json
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def stream_hash(b: bytes) -> str:
    if len(b) >= 16:
        b = b[:12] + b"\0\0\0\0" + b[16:]
    return hashlib.sha256(b).hexdigest()


def file_hash(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def parse_meta(b: bytes):
    name_len, n = struct.unpack_from("<ii", b, 0)
    ebs = list(struct.unpack_from("<%df" % n, b, 8))
    (rng,) = struct.unpack_from("<f", b, 8 + 4 * n)
    name = b[12 + 4 * n: 12 + 4 * n + name_len].decode("utf-8", "replace")
    return {"ebs": [struct.unpack("<I", struct.pack("<f", e))[0] for e in ebs],
            "range": struct.unpack("<I", struct.pack("<f", rng))[0], "name": os.path.basename(name)}


def main(root):
    out = {}
    for case in sorted(os.listdir(root)):
        cdir = os.path.join(root, case)
        if not os.path.isdir(cdir):
            continue
        for mode in sorted(os.listdir(cdir)):
            d = os.path.join(cdir, mode)
            rec = {"rc": {}}
            for line in open(os.path.join(d, "rc.txt")):
                k, v = line.split()
                rec["rc"][k] = int(v)
            sdir = os.path.join(d, "stor")
            if os.path.isdir(sdir):
                stor = {}
                for f in sorted(os.listdir(sdir)):
                    b = open(os.path.join(sdir, f), "rb").read()
                    if f == ".stor.meta":
                        rec["meta"] = parse_meta(b)
                    else:
                        stor[f.rsplit(".", 1)[1]] = {"sha256": stream_hash(b), "bytes": len(b)}
                rec["stor"] = stor
            for f, kind in (("init.bin", "s"), ("resi.bin", "s"), ("init_dec.f32", "f"), ("resi_dec.f32", "f")):
                p = os.path.join(d, f)
                if os.path.exists(p):
                    b = open(p, "rb").read()
                    rec[f] = {"sha256": stream_hash(b) if kind == "s" else file_hash(b), "bytes": len(b)}
            for log in ("store_bench", "init_bench", "resi_bench"):
                p = os.path.join(d, log + ".log")
                if os.path.exists(p):
                    t = open(p).read()
                    rec[log + "_verify"] = ("ERROR" not in t) and ("verification passed" in t or log == "store_bench")
            out[f"{case}/{mode}"] = rec
    with open(os.path.join(HERE, "reference_outputs.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("collected", len(out), "runs")


if __name__ == "__main__":
    main(sys.argv[1])
