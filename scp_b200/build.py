"""In-tree build of libscpgpu.so for sm_100a (``python -m scp_b200.build``).

nvcc cross-compiles without a GPU; the shared object lands next to this file
so it travels with the source tree.  The CUDA runtime is linked statically.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-v"]
SOURCES = [os.path.join(HERE, "csrc", "scp_gpu.cu")]
OUT = os.path.join(HERE, "libscpgpu.so")


def _deps() -> list[str]:
    d = os.path.join(HERE, "csrc")
    return SOURCES + [os.path.join(d, f) for f in os.listdir(d)] + [os.path.join(ROOT, "include", "scp_gpu.h")]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    cmd = [NVCC, *ARCH, *FLAGS, "-I", os.path.join(ROOT, "include"), "-o", OUT, *SOURCES]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libscpgpu.so")
    if verbose:
        sys.stderr.write(res.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
