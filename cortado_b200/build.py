"""Builds libcortado.so and the five command-line drivers in-tree with nvcc
for sm_100a (no JIT cache, so the binaries travel with the source tree)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcortado.so")
BIN = os.path.join(HERE, "bin")
CLIS = {"store": "CLI_STORE", "init_send": "CLI_INIT_SEND", "init_recv": "CLI_INIT_RECV",
        "resi_send": "CLI_RESI_SEND", "resi_recv": "CLI_RESI_RECV"}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


def deps():
    out = [os.path.join(ROOT, "include", "cortado.h"), os.path.join(HERE, "cli", "cortado_cli.c")]
    out += [os.path.join(SRC, f) for f in os.listdir(SRC)]
    return out


def _stale(target) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(f) > t for f in deps())


def build(force: bool = False, verbose: bool = False, clis: bool = True) -> str:
    targets = [LIB] + ([os.path.join(BIN, c) for c in CLIS] if clis else [])
    if not (force or any(_stale(t) for t in targets)):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    obj = os.path.join(BUILD, "cortado.o")
    cmd = ["nvcc", *NVCC_FLAGS, "-c", "-o", obj, os.path.join(SRC, "cortado.cu")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.check_call(cmd)
    subprocess.check_call(["nvcc", *ARCH, "-shared", "-o", LIB, obj])
    if clis:
        os.makedirs(BIN, exist_ok=True)
        for name, macro in CLIS.items():
            cobj = os.path.join(BUILD, f"cli_{name}.o")
            subprocess.check_call(["nvcc", *ARCH, "-O2", f"-D{macro}", "-c", "-o", cobj, os.path.join(HERE, "cli", "cortado_cli.c")])
            subprocess.check_call(["nvcc", *ARCH, "-o", os.path.join(BIN, name), cobj, obj])
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
