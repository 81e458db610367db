"""Builds the sm_100a CUDA library in-tree: uncertaintea_b200/libut_b200.so.

The C ABI and its kernels are compiled by nvcc for sm_100a only, from
csrc/ut_api.cu, csrc/ut_noalloc.cu (the allocation-free entry point, whose
kernels are private to its file), csrc/ut_surrogate.cu (the learned
gradient surrogate) and csrc/ut_multi.cu (many models in one batched launch),
each in its own process, then linked into one shared library.  Run: python -m uncertaintea_b200.build [--force]
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libut_b200.so")
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH_FLAGS + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                           "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh"))
                  + [os.path.join(ROOT, "include", "ut_b200.h")])


UNITS = ["ut_api.cu", "ut_noalloc.cu", "ut_surrogate.cu", "ut_multi.cu"]


def build(force: bool = False, verbose: bool = False) -> str:
    newest = max(os.path.getmtime(s) for s in sources())
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    # each translation unit compiles in its own nvcc process (the kernel
    # template instantiations make ut_api.cu the longest), then one link
    import concurrent.futures as cf
    objs = [os.path.join(HERE, "csrc", u[:-3] + ".o") for u in UNITS]
    flags = [f for f in NVCC_FLAGS if f != "-shared"] + (["-Xptxas=-v"] if verbose else [])

    def compile_unit(i):
        subprocess.run([nvcc()] + flags + ["-c", "-o", objs[i], os.path.join(HERE, "csrc", UNITS[i])], check=True)

    with cf.ThreadPoolExecutor(len(UNITS)) as pool:
        list(pool.map(compile_unit, range(len(UNITS))))
    subprocess.run([nvcc()] + ARCH_FLAGS + ["-shared", "-o", LIB + ".tmp"] + objs, check=True)
    os.replace(LIB + ".tmp", LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
