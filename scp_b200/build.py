"""In-tree build of libscpgpu.so for sm_100a (``python -m scp_b200.build``).

nvcc cross-compiles without a GPU; the shared object lands next to this file
so it travels with the source tree.  The CUDA runtime is linked statically.
Each translation unit compiles in its own nvcc process (objects under
scp_b200/_build/), then one nvcc call links the shared object.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v"]
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("scp_gpu.cu", "kern_f64.cu", "kern_f32c.cu", "kern_pair.cu", "kern_ext.cu", "kern_tma.cu", "kern_duo.cu")]
OUT = os.path.join(HERE, "libscpgpu.so")
OBJDIR = os.path.join(HERE, "_build")


def _deps() -> list[str]:
    d = os.path.join(HERE, "csrc")
    return SOURCES + [os.path.join(d, f) for f in os.listdir(d)] + [os.path.join(ROOT, "include", "scp_gpu.h")]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(f) <= t for f in _deps())


def _compile(src: str) -> tuple[str, subprocess.CompletedProcess]:
    obj = os.path.join(OBJDIR, os.path.basename(src).replace(".cu", ".o"))
    cmd = [NVCC, *ARCH, *FLAGS, "-I", os.path.join(ROOT, "include"), "-c", "-o", obj, src]
    return obj, subprocess.run(cmd, capture_output=True, text=True)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(OBJDIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(_compile, SOURCES))
    for src, (obj, res) in zip(SOURCES, results):
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError(f"nvcc failed on {os.path.basename(src)}")
        if verbose:
            sys.stderr.write(res.stderr)
    res = subprocess.run([NVCC, *ARCH, "-shared", "-o", OUT, *[o for o, _ in results]], capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed linking libscpgpu.so")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
