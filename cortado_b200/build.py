"""Builds libcortado.so in-tree with nvcc for sm_100a (no JIT cache, so the
library travels with the source tree)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcortado.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def sources():
    return [os.path.join(SRC, "cortado.cu")]


def deps():
    out = [os.path.join(ROOT, "include", "cortado.h")]
    for f in os.listdir(SRC):
        out.append(os.path.join(SRC, f))
    return out


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if force or stale():
        cmd = ["nvcc", *NVCC_FLAGS, "-o", LIB, *sources()]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
