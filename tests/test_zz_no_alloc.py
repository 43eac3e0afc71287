"""The allocation-free energy entry point (ems_energy_noalloc) against the
engine's own energy.

Some callers of this library cannot allocate device memory at the moment
they need a result: a host whose framework owns all device memory through
its own pool, or a real-time loop that must not allocate once started.
ems_energy_noalloc serves them: it takes the caller's device arrays and a
caller-provided device double and uses only a fixed 16 KiB device array of
the library as working memory. This file is collected last (test_zz_) so a
run that stops at its first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

import ems_b200 as E
from ems_b200 import workloads as W

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the energy tolerance of the other parity tests (a reduction)


def _noalloc(model, fields, coeff, out, stream):
    lib = E.gpu_lib()
    nodes = (C.c_uint64 * 3)(*model.nodes)
    u = (C.c_void_p * 3)(*[t.data_ptr() for t in fields[:3]])
    i = (C.c_void_p * 3)(*[t.data_ptr() for t in fields[3:]])
    co = (C.c_void_p * 12)(*[t.data_ptr() for t in coeff])
    return lib.ems_energy_noalloc(nodes, model.dt, u, i, co, C.c_void_p(out.data_ptr()), C.c_void_p(stream))


def test_energy_noalloc_equals_step_with_energy():
    import torch

    w = W.vacuum_box(n=24, cpml=4, steps=400, f0=10e9, fc=8e9)
    m = w.model
    g = E.Engine(m, device=0)
    coeff = [torch.from_numpy(np.ascontiguousarray(m.coeff(l))).to("cuda:0") for l in range(12)]
    stream = torch.cuda.current_stream(0).cuda_stream
    g.run(40)
    for _ in range(2):
        fields = [torch.from_numpy(g.field(f, a)).to("cuda:0") for f in (0, 1) for a in range(3)]
        got = []
        for _call in range(2):  # two calls in a row share the scratch array
            out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda:0")
            assert _noalloc(m, fields, coeff, out, stream) == 0
            torch.cuda.synchronize(0)
            got.append(out.item())
        # The engine's energy of the same state (the state before its next
        # step; CPML, source and probes hold no energy).
        want = g.step_with_energy()
        assert want > 0.0
        for x in got:
            assert abs(x - want) <= RTOL * abs(want), (x, want)
        assert got[0] == got[1]
        g.run(13)


def test_energy_noalloc_rejects_sizes_beyond_its_limit():
    import torch

    lib = E.gpu_lib()
    t = torch.zeros(8, device="cuda:0")
    ptrs3 = (C.c_void_p * 3)(*[t.data_ptr()] * 3)
    ptrs12 = (C.c_void_p * 12)(*[t.data_ptr()] * 12)
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    big = (C.c_uint64 * 3)(2048, 2048, 1024)  # 2^32 nodes: beyond 2^31 − 1
    assert lib.ems_energy_noalloc(big, 1e-12, ptrs3, ptrs3, ptrs12, C.c_void_p(out.data_ptr()), None) == 1
    # A product that wraps in 64 bits to under 2^31 − 1: rejected too.
    wrap = (C.c_uint64 * 3)(131073, 65537, 2147434497)
    assert lib.ems_energy_noalloc(wrap, 1e-12, ptrs3, ptrs3, ptrs12, C.c_void_p(out.data_ptr()), None) == 1
    small = (C.c_uint64 * 3)(1, 2, 2)
    assert lib.ems_energy_noalloc(small, 1e-12, ptrs3, ptrs3, ptrs12, C.c_void_p(out.data_ptr()), None) == 1
