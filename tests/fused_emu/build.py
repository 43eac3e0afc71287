"""Builds the CPU emulation of the fused step kernel (test infrastructure)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def build(asan: bool = False) -> str:
    out = os.path.join(HERE, "libfused_emu_asan.so" if asan else "libfused_emu.so")
    deps = [os.path.join(HERE, f) for f in ("harness.cpp", "emu_shim.h")] + [
        os.path.join(ROOT, "ems_b200", "csrc", f) for f in ("fused.cuh", "kernels.cuh", "arith.cuh", "separate.cuh", "split.cuh", "interior.cuh", "march.cuh", "fused_tables.h")]
    if os.path.exists(out) and all(os.path.getmtime(d) <= os.path.getmtime(out) for d in deps):
        return out
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-ffp-contract=off", "-fPIC", "-shared", "-DEMS_HOST_EMULATION",
           "-Wno-format-truncation", "-I", os.path.join(ROOT, "include"), "-o", out + ".tmp",
           os.path.join(HERE, "harness.cpp"), "-lpthread"]
    if asan:
        cmd[1:1] = ["-fsanitize=address", "-fno-omit-frame-pointer"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    os.replace(out + ".tmp", out)
    return out
