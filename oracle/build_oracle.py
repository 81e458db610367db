"""Build recipe of the CPU oracle (test infrastructure only).

Compiles oracle/oracle.cpp, oracle/oracle_mlp.cpp and oracle/oracle_program.cpp into
oracle/_build/liboracle.so with g++ and OpenMP.  Run: python oracle/build_oracle.py
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, "oracle.cpp"), os.path.join(HERE, "oracle_mlp.cpp"), os.path.join(HERE, "oracle_program.cpp")]
    deps = srcs + [os.path.join(HERE, "oracle_mlp.h"), os.path.join(HERE, "oracle_program.h"),
                   os.path.join(HERE, "..", "include", "ut_b200.h")]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared"] + srcs + ["-o", LIB]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
