"""Builds libfemh.so (sm_100a) in-tree with nvcc.

The library is the product: C++ host code plus hand-written CUDA kernels
behind the C ABI of include/femh.h.  No torch, no JIT cache: the .so lands in
fem_b200/ so that it travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfemh.so")
SOURCES = [os.path.join(CSRC, "engine.cu"), os.path.join(HERE, "host", "femh_host.cpp")]
HEADERS = [os.path.join(CSRC, f) for f in ("femh_common.cuh", "stencil.cuh", "kernels.cuh")] + [
    os.path.join(HERE, "host", "femh_host.hpp")]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3",
    "--expt-relaxed-constexpr",
    "-shared",
    "-ccbin", "g++",
]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = SOURCES + HEADERS + [os.path.join(ROOT, "include", "femh.h"), os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    if not force and not _stale():
        return LIB
    cmd = [NVCC, *FLAGS, "-o", LIB, *SOURCES, "-lcudart"]
    if ptxas_v:
        cmd.insert(1, "-Xptxas=-v")
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    res = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True, env=env)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if verbose or ptxas_v:
        sys.stderr.write(res.stdout + res.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_v="--ptxas" in sys.argv)
