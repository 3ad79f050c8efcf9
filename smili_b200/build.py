"""Build the in-tree CUDA libraries with nvcc for sm_100a.

``libsmili_b200.so``: the imaging solver (solver.cu and its headers).
``libsmili_unet.so``: the BF16 kernels of the warm-start U-Net (unet.cu).
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
INC = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "-diag-suppress", "177"]

# output -> (main source, dependencies under csrc/, headers under include/)
LIBS = {
    "libsmili_b200.so": ("solver.cu", ["common.cuh", "fft.cuh", "fg.cuh", "lbfgsb.cuh", "layout.h", "uvlist.cuh"],
                         ["smili_b200.h"]),
    "libsmili_unet.so": ("unet.cu", ["conv_tc.cuh"], ["smili_unet.h"]),
}

OUT = os.path.join(HERE, "libsmili_b200.so")
UNET_OUT = os.path.join(HERE, "libsmili_unet.so")


def _stale(out: str, src: str, deps, hdrs) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    files = [os.path.join(HERE, "csrc", f) for f in [src] + list(deps)]
    files += [os.path.join(INC, h) for h in hdrs]
    return any(os.path.getmtime(f) > t for f in files)


def build_one(name: str, force: bool = False, verbose: bool = False) -> str:
    src, deps, hdrs = LIBS[name]
    out = os.path.join(HERE, name)
    if force or _stale(out, src, deps, hdrs):
        nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
        cmd = [nvcc] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + \
            ["-o", out, os.path.join(HERE, "csrc", src)]
        subprocess.run(cmd, check=True)
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    """Build every library; returns the solver library's path."""
    for name in LIBS:
        build_one(name, force, verbose)
    return OUT


if __name__ == "__main__":
    build(force=True, verbose=True)
