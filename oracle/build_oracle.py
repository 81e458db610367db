"""Build recipe of the CPU oracle (test infrastructure only).

Compiles oracle/oracle.cpp into oracle/_build/liboracle.so with g++ and
OpenMP.  Run: python oracle/build_oracle.py
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "oracle.cpp")
    hdr = os.path.join(HERE, "..", "include", "ut_b200.h")
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(src), os.path.getmtime(hdr)):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", src, "-o", LIB]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
