"""Builds libamoeba_gpu.so in-tree for sm_100a with nvcc (no JIT cache):

    python -m polmdqc_b200.build

The library lands in polmdqc_b200/_lib/ so that it travels with the source
tree; `-Xptxas -v` output (registers, spills) is kept in _lib/ptxas.log.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libamoeba_gpu.so")
SOURCES = ["amg_api.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "amoeba_gpu.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-v", "-I", os.path.join(ROOT, "include"),
           *[os.path.join(CSRC, s) for s in SOURCES], "-o", LIB, "-lcufft"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    with open(os.path.join(OUT_DIR, "ptxas.log"), "w") as f:
        f.write(proc.stdout + proc.stderr)
    if proc.returncode != 0:
        sys.stderr.write(proc.stderr[-6000:])
        raise RuntimeError("nvcc failed building libamoeba_gpu.so")
    if verbose:
        print(proc.stderr[-3000:])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
