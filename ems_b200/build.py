"""Builds the engine's shared libraries in-tree.

* ``ems_b200/libems_gpu.so``  — the CUDA engine (include/ems_gpu.h), sm_100a;
* ``ems_b200/libems_host.so`` — host-side set-up and run loop (include/ems_host.h);
* ``ems_b200/libems_learn.so`` — the learned early stop's kernels (include/ems_learn.h).

The CUDA sources are compiled without fused multiply-add contraction and
with IEEE denormals, division and square root, which the engine's bit-exact
arithmetic relies on. ``python -m ems_b200.build`` rebuilds what is stale.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-ftz=false", "-prec-div=true",
    "-prec-sqrt=true", "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared",
]
CXX_FLAGS = ["-O3", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-Wall", "-Wextra"]

GPU_LIB = os.path.join(HERE, "libems_gpu.so")
HOST_LIB = os.path.join(HERE, "libems_host.so")
LEARN_LIB = os.path.join(HERE, "libems_learn.so")


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {' '.join(cmd)}")


def build_gpu(force: bool = False) -> str:
    srcs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cuh", ".h")) or f in ("engine.cu", "noalloc.cu")]
    srcs += [os.path.join(INCLUDE, "ems_gpu.h")]
    if force or _stale(GPU_LIB, srcs):
        tmp = GPU_LIB + ".tmp"
        _run([_nvcc(), *NVCC_ARCH, *NVCC_FLAGS, "-I", INCLUDE, "-o", tmp, os.path.join(CSRC, "engine.cu"),
              os.path.join(CSRC, "noalloc.cu")])
        os.replace(tmp, GPU_LIB)
    return GPU_LIB


def build_learn(force: bool = False) -> str:
    """The learned early stop's kernels (include/ems_learn.h)."""
    srcs = [os.path.join(CSRC, "learn.cu"), os.path.join(INCLUDE, "ems_learn.h")]
    if force or _stale(LEARN_LIB, srcs):
        tmp = LEARN_LIB + ".tmp"
        _run([_nvcc(), *NVCC_ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-I", INCLUDE,
              "-o", tmp, os.path.join(CSRC, "learn.cu")])
        os.replace(tmp, LEARN_LIB)
    return LEARN_LIB


def build_host(force: bool = False) -> str:
    srcs = [os.path.join(CSRC, "host.cpp"), os.path.join(INCLUDE, "ems_host.h"), os.path.join(INCLUDE, "ems_gpu.h")]
    if force or _stale(HOST_LIB, srcs):
        tmp = HOST_LIB + ".tmp"
        _run(["g++", *CXX_FLAGS, "-I", INCLUDE, "-o", tmp, os.path.join(CSRC, "host.cpp"), "-lpthread"])
        os.replace(tmp, HOST_LIB)
    return HOST_LIB


def build(force: bool = False) -> None:
    build_host(force)
    build_gpu(force)
    build_learn(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(HOST_LIB)
    print(GPU_LIB)
    print(LEARN_LIB)
