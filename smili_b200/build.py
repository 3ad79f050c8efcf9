"""Build ``libsmili_b200.so`` in-tree with nvcc for sm_100a."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "solver.cu")
OUT = os.path.join(HERE, "libsmili_b200.so")
DEPS = ["solver.cu", "common.cuh", "fft.cuh", "fg.cuh", "lbfgsb.cuh", "layout.h"]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "-diag-suppress", "177"]


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    hdr = os.path.join(os.path.dirname(HERE), "include", "smili_b200.h")
    return any(os.path.getmtime(os.path.join(HERE, "csrc", f)) > t for f in DEPS) or \
        os.path.getmtime(hdr) > t


def build(force: bool = False, verbose: bool = False) -> str:
    if force or _stale():
        nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
        cmd = [nvcc] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", OUT, SRC]
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force=True, verbose=True)
