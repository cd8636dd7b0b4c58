"""Build the in-tree CUDA library ``higflow_b200/lib/libhigflow_b200.so``.

nvcc compiles for sm_100a only.  The kernels that restate the reference's
arithmetic are compiled with ``-fmad=false`` so the FP64 form keeps the
reference's rounding sequence (no fused multiply-add contraction).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "lib", "libhigflow_b200.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("hf_engine.cu", "hf_server.cpp")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", f) for f in ("hf_device.cuh", "hf_amg.cuh", "hf_pcg.cuh")] + \
    [os.path.join(REPO, "include", "higflow_b200.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-fmad=false",
    "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-I" + os.path.join(REPO, "include"),
]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = [nvcc()] + NVCC_FLAGS + SOURCES + ["-o", LIB]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
