"""Builds the sm_100a CUDA library in-tree: uncertaintea_b200/libut_b200.so.

The C ABI and its kernels are compiled by nvcc for sm_100a only, from
csrc/ut_api.cu, csrc/ut_noalloc.cu (the allocation-free entry point, whose
kernels are private to its file), csrc/ut_surrogate.cu (the learned
gradient surrogate) and csrc/ut_multi.cu (many models in one batched launch).  Run: python -m uncertaintea_b200.build [--force]
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


def build(force: bool = False, verbose: bool = False) -> str:
    newest = max(os.path.getmtime(s) for s in sources())
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", LIB + ".tmp", os.path.join(HERE, "csrc", "ut_api.cu"),
                                   os.path.join(HERE, "csrc", "ut_noalloc.cu"),
                                   os.path.join(HERE, "csrc", "ut_surrogate.cu"),
                                   os.path.join(HERE, "csrc", "ut_multi.cu")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
