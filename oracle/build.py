"""Builds the oracle (test infrastructure): ``oracle/liboracle.so``.

The oracle is the CPU restatement of the reference engine's step that the
tests compare the CUDA engine with and that ``bench.py`` times as the CPU
baseline. It is compiled without floating-point contraction so its f32/f64
arithmetic is the reference's, operation by operation.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRCS = [os.path.join(HERE, "oracle.cpp")]
DEPS = SRCS + [os.path.join(HERE, "oracle.h"), os.path.join(os.path.dirname(HERE), "include", "ems_gpu.h")]


def build(force: bool = False) -> str:
    stale = force or not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in DEPS)
    if stale:
        tmp = LIB + ".tmp"
        cmd = ["g++", "-O3", "-march=x86-64-v3", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared",
               "-Wall", "-Wextra", "-o", tmp, *SRCS, "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("oracle build failed")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
