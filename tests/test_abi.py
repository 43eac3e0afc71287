"""The C-ABI libraries load and export every symbol their headers declare
(no compute calls: these run without a GPU)."""
import ctypes as C
import os
import re

import pytest

import ems_b200 as E

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header: str) -> list[str]:
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(ems_[a-z0-9_]+)\s*\(", src)
    return sorted(set(n for n in names if not n.endswith("_t")))


def test_gpu_header_symbols_exported():
    from ems_b200 import build

    path = build.build_gpu()
    lib = C.CDLL(path)  # loads without a device: no CUDA call at load time
    names = declared("ems_gpu.h")
    assert "ems_gpu_create" in names and "ems_gpu_run" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # The Python binding covers the whole header.
    assert set(names) == set(E.GPU_SYMBOLS)


def test_host_header_symbols_exported():
    lib = E.host_lib()
    names = declared("ems_host.h")
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_oracle_exports():
    import oracle

    lib = oracle.lib()
    for n in ("oracle_create", "oracle_run", "oracle_step_with_energy", "oracle_samples"):
        assert hasattr(lib, n)


def test_null_arguments_are_rejected_without_a_device():
    lib = E.gpu_lib()
    h = C.c_void_p()
    assert lib.ems_gpu_create(None, 0, C.byref(h)) == 1  # EMS_ERR_INVALID
    assert lib.ems_gpu_run(None, 1) == 1
    assert lib.ems_gpu_destroy(None) == 1
    assert lib.ems_gpu_last_error(None) == b"null handle"


def test_noalloc_size_checks_without_a_device():
    """ems_energy_noalloc validates its sizes before any CUDA call, so the
    refusals run here: a node count beyond 2^31 − 1, one whose product wraps
    in 64 bits to a small number, and a dimension under 2."""
    lib = E.gpu_lib()
    dummy = (C.c_float * 4)()
    p3 = (C.c_void_p * 3)(*[C.addressof(dummy)] * 3)
    p12 = (C.c_void_p * 12)(*[C.addressof(dummy)] * 12)
    out = C.c_double()
    for dims in [(2048, 2048, 1024), (131073, 65537, 2147434497), (2**63, 2**62, 8), (1, 2, 2)]:
        nodes = (C.c_uint64 * 3)(*dims)
        assert lib.ems_energy_noalloc(nodes, 1e-12, p3, p3, p12, C.byref(out), None) == 1, dims


def test_gpu_library_is_sm100a():
    """The engine is compiled for sm_100a only (no other SASS or PTX)."""
    from ems_b200 import build

    assert "arch=compute_100a,code=sm_100a" in " ".join(build.NVCC_ARCH)
    assert "--fmad=false" in build.NVCC_FLAGS


@pytest.mark.parametrize("header", ["ems_gpu.h", "ems_host.h"])
def test_headers_compile_as_c(header, tmp_path):
    import subprocess

    src = tmp_path / "t.c"
    src.write_text(f'#include "{header}"\nint main(void) {{ return 0; }}\n')
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                        "-o", str(tmp_path / "t")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
