"""Build libisinggpu.so in-tree with nvcc for sm_100a.

The library is the product: CUDA kernels, the host lattice compiler and the C-ABI of
include/ising_gpu.h.  It is compiled explicitly (no JIT cache) so the shared object sits
next to this file and travels with the source tree.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libisinggpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]
    for c in cand:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
                  + glob.glob(os.path.join(HERE, "..", "include", "*.h")))


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in sources() + headers())


BUILD_DIR = os.path.join(HERE, "_build")


def _compile(src: str, obj: str, extra) -> None:
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-c",
           "-ccbin", shutil.which("g++") or "g++",
           "-I", os.path.join(HERE, "..", "include"), *extra, "-o", obj + ".tmp", src]
    subprocess.run(cmd, check=True)
    os.replace(obj + ".tmp", obj)


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    """Compile every source to an object in _build/ (in parallel; a source is recompiled
    when it or any header is newer than its object), then link libisinggpu.so."""
    if not force and not needs_build():
        return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    newest_header = max((os.path.getmtime(h) for h in headers()), default=0.0)
    jobs = []
    objs = []
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), newest_header):
            jobs.append((src, obj))
    if verbose:
        print(f"compiling {len(jobs)} of {len(objs)} sources", file=sys.stderr)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_compile, src, obj, list(extra)) for src, obj in jobs]:
            f.result()
    cmd = [nvcc(), *ARCH, "-shared", "-ccbin", shutil.which("g++") or "g++", "-o", LIB + ".tmp", *objs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else [])
    print(LIB)
