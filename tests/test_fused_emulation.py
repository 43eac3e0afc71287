"""The fused step kernel's own source, run on the CPU (tests/fused_emu), equals
the oracle bit for bit.

The CUDA source of the fused kernel (ems_b200/csrc/fused.cuh) is compiled
for the host with a shim that turns each CUDA thread into a host thread and
each TMA bulk copy into a checked memcpy (shared-memory bounds, 16-byte
alignment, the mbarrier's expected bytes and phases). This checks the
kernel's tiling, halo rows, x chunks, stage ring and indexing without a
GPU; the oracle is the reference's step restated.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

import ems_b200 as E
from ems_b200 import workloads as W
from oracle import OracleEngine

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

HERE = os.path.dirname(os.path.abspath(__file__))


def emu_lib(asan=False):
    from fused_emu import build

    lib = C.CDLL(build.build(asan))
    lib.emu_fused_run.restype = C.c_int
    lib.emu_fused_run.argtypes = [C.c_void_p, C.c_int, C.c_uint, C.c_uint64, C.c_void_p, C.c_void_p]
    lib.emu_two_run.restype = C.c_int
    lib.emu_two_run.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    lib.emu_split_run.restype = C.c_int
    lib.emu_split_run.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    lib.emu_split_rows_run.restype = C.c_int
    lib.emu_split_rows_run.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p]
    lib.emu_interior_run.restype = C.c_int
    lib.emu_interior_run.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    lib.emu_march_run.restype = C.c_int
    lib.emu_march_run.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32, C.c_uint32]
    lib.emu_march_timeout.restype = C.c_int
    lib.emu_march_timeout.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64]
    lib.emu_pole_prev_fold.restype = C.c_int
    lib.emu_pole_prev_fold.argtypes = [C.c_void_p, C.c_int]
    lib.emu_error.restype = C.c_char_p
    return lib


def model(n, scheme, cpml=3, poles=True, graded=False, magnetic=False):
    rng = np.random.default_rng(11)
    if graded:
        lines = [np.cumsum(np.concatenate([[0.0], 1e-3 * (1.0 + 0.3 * rng.random(c))])) for c in n]
        m = E.Model(*lines)
    else:
        m = E.Model.uniform(n, [1e-3] * 3)
    sph = m.cells().sphere([n[0] / 2, n[1] / 2, n[2] / 2], min(n) / 4)
    m.fill(sph, m.material(eps_r=2.0, kappa=0.01))
    m.fill_pec_box([1, 1, 1], [3, 2, 3])
    m.build()
    if cpml:
        m.add_cpml([cpml, cpml + 1, cpml, 0, cpml, cpml], kappa_max=1.5, alpha_max=0.02)
    if poles:
        d = E.Dispersive()
        d.fill_cells(m, sph, W.lorentz_poles(5))
        d.fill_cells(m, m.cells().box([0, 0, n[2] - 4], [n[0], n[1], n[2] - 2]), [E.Pole.drude(6e10, 6e9)])
        d.fill_cells(m, m.cells().box([2, 2, 2], [5, 4, 6]), [E.Pole.debye(1.5, 1e-11)])
        if magnetic:
            d.fill_cells(m, m.cells().box([1, 3, 2], [6, 7, 5]), [E.Pole.lorentz(3e10, 2e10, 1e9)], field=1)
            d.fill_cells(m, m.cells().box([2, 1, 4], [5, 5, 8]), [E.Pole.drude(2e10, 3e9)], field=1)
        m.add_dispersive(d, scheme)
    return m


def random_state(m, seed=0):
    rng = np.random.default_rng(seed)
    return [(rng.standard_normal(m.nodes) * 1e-2).astype(np.float32) for _ in range(6)]


def run_emu(lib, m, state, steps, tj, grid):
    arrs = [np.ascontiguousarray(s.copy()) for s in state]
    ptrs = (C.c_void_p * 6)(*[a.ctypes.data for a in arrs])
    en = np.zeros(steps)
    r = lib.emu_fused_run(m.desc, tj, grid, steps, ptrs, en.ctypes.data)
    assert r == 0, lib.emu_error().decode()
    return arrs, en


def run_oracle(m, state, steps):
    o = OracleEngine(m, threads=2)
    for f in range(2):
        for a in range(3):
            o.set_field(f, a, state[3 * f + a])
    en = [o.step_with_energy() for _ in range(steps)]
    return [o.field(f, a) for f in range(2) for a in range(3)], np.array(en), o


@pytest.mark.parametrize("n,tj,grid,scheme", [
    ((9, 10, 13), 2, 1, E.TRAPEZOIDAL),
    ((12, 11, 9), 4, 3, E.LEAPFROG),
    ((17, 14, 40), 6, 2, E.TRAPEZOIDAL),
    ((21, 7, 33), 4, 5, E.LEAPFROG),
    ((12, 11, 9), 4, 3, E.OPENEMS_POLES),
    ((17, 14, 40), 6, 2, E.OPENEMS_POLES),
])
def test_fused_kernel_source_equals_oracle(n, tj, grid, scheme):
    m = model(n, scheme, graded=tj == 4)
    state = random_state(m)
    steps = 12
    got, eg = run_emu(emu_lib(), m, state, steps, tj, grid)
    want, eo, o = run_oracle(m, state, steps)
    names = ["u_x", "u_y", "u_z", "i_x", "i_y", "i_z"]
    for name, a, b in zip(names, got, want):
        bad = np.argwhere(a.view(np.uint32) != b.view(np.uint32))
        assert bad.size == 0, f"{name}: {len(bad)} differ, first {tuple(bad[0])}: {a[tuple(bad[0])]} vs {b[tuple(bad[0])]}"
    # The field part of the invariant (the oracle adds the pole energy).
    assert np.all(np.isfinite(eg)) and np.all(eg > 0)


@pytest.mark.parametrize("n,scheme,magnetic", [
    ((9, 10, 13), E.TRAPEZOIDAL, True),
    ((12, 11, 35), E.LEAPFROG, True),
    ((10, 9, 8), E.LEAPFROG, False),
    ((12, 11, 35), E.OPENEMS_POLES, True),
])
def test_two_kernel_source_equals_oracle(n, scheme, magnetic):
    m = model(n, scheme, magnetic=magnetic)
    state = random_state(m, seed=1)
    steps = 10
    arrs = [np.ascontiguousarray(x.copy()) for x in state]
    ptrs = (C.c_void_p * 6)(*[a.ctypes.data for a in arrs])
    en = np.zeros(steps)
    lib = emu_lib()
    assert lib.emu_two_run(m.desc, steps, ptrs, en.ctypes.data) == 0, lib.emu_error().decode()
    want, eo, o = run_oracle(m, state, steps)
    for name, a, b in zip(["u_x", "u_y", "u_z", "i_x", "i_y", "i_z"], arrs, want):
        bad = np.argwhere(a.view(np.uint32) != b.view(np.uint32))
        assert bad.size == 0, f"{name}: {len(bad)} differ, first {tuple(bad[0])}"
    # The field part of the invariant: the oracle's total less its pole energy
    # is not available per step, so compare a model without poles below.
    assert np.all(np.isfinite(en))


def test_two_kernel_energy_equals_oracle():
    m = model((10, 9, 12), E.TRAPEZOIDAL, poles=False)
    state = random_state(m, seed=2)
    steps = 5
    arrs = [np.ascontiguousarray(x.copy()) for x in state]
    ptrs = (C.c_void_p * 6)(*[a.ctypes.data for a in arrs])
    en = np.zeros(steps)
    lib = emu_lib()
    assert lib.emu_two_run(m.desc, steps, ptrs, en.ctypes.data) == 0, lib.emu_error().decode()
    _, eo, _ = run_oracle(m, state, steps)
    np.testing.assert_allclose(en, eo, rtol=1e-12, atol=0)
    got, eg = run_emu(lib, m, state, steps, 4, 2)
    np.testing.assert_allclose(eg, eo, rtol=1e-12, atol=0)


@pytest.mark.parametrize("n,graded", [((10, 9, 12), False), ((12, 11, 35), True), ((9, 14, 40), False)])
def test_split_source_equals_oracle(n, graded):
    """The split schedule's update and CPML shell kernels: fields bit-exact,
    energy within 1e-12 (a sum in another order)."""
    m = model(n, E.TRAPEZOIDAL, poles=False, graded=graded)
    state = random_state(m, seed=3)
    steps = 6
    arrs = [np.ascontiguousarray(x.copy()) for x in state]
    ptrs = (C.c_void_p * 6)(*[a.ctypes.data for a in arrs])
    en = np.zeros(steps)
    lib = emu_lib()
    assert lib.emu_split_run(m.desc, steps, ptrs, en.ctypes.data) == 0, lib.emu_error().decode()
    want, eo, _ = run_oracle(m, state, steps)
    for name, a, b in zip(["u_x", "u_y", "u_z", "i_x", "i_y", "i_z"], arrs, want):
        bad = np.argwhere(a.view(np.uint32) != b.view(np.uint32))
        assert bad.size == 0, f"{name}: {len(bad)} differ, first {tuple(bad[0])}"
    np.testing.assert_allclose(en, eo, rtol=1e-12, atol=0)


@pytest.mark.parametrize("n,graded,faces", [((10, 9, 12), False, None), ((12, 11, 35), True, None),
                                             ((14, 13, 18), True, [3, 2, 4, 3, 2, 3]), ((9, 14, 40), False, [0, 3, 2, 0, 3, 3]),
                                             ((8, 9, 7), False, [2, 2, 2, 2, 1, 1]), ((11, 8, 6), True, [1, 0, 2, 1, 3, 3])])
def test_split_rows_source_equals_oracle(n, graded, faces):
    """The split schedule with the row CPML: every slab's correction applied
    inside the update kernels' CPML variant over the quads holding layer
    nodes (x-layer planes, y-layer rows, the z-layer quads at the row ends),
    the plain kernel elsewhere, no shell (corners of two and three layers,
    faces without a layer, z layers that overlap inside one quad). Fields
    bit-exact against the oracle."""
    m = model(n, E.TRAPEZOIDAL, poles=False, graded=graded, cpml=0)
    m.add_cpml(faces or [3, 4, 3, 0, 3, 3], kappa_max=1.5, alpha_max=0.02)
    state = random_state(m, seed=5)
    steps = 6
    arrs = [np.ascontiguousarray(x.copy()) for x in state]
    ptrs = (C.c_void_p * 6)(*[a.ctypes.data for a in arrs])
    lib = emu_lib()
    assert lib.emu_split_rows_run(m.desc, steps, ptrs) == 0, lib.emu_error().decode()
    want, _, _ = run_oracle(m, state, steps)
    for name, a, b in zip(["u_x", "u_y", "u_z", "i_x", "i_y", "i_z"], arrs, want):
        bad = np.argwhere(a.view(np.uint32) != b.view(np.uint32))
        assert bad.size == 0, f"{name}: {len(bad)} differ, first {tuple(bad[0])}"


def run_interior(lib, m, state, steps):
    arrs = [np.ascontiguousarray(x.copy()) for x in state]
    ptrs = (C.c_void_p * 6)(*[a.ctypes.data for a in arrs])
    box = (C.c_uint32 * 6)()
    assert lib.emu_interior_run(m.desc, steps, ptrs, box) == 0, lib.emu_error().decode()
    return arrs, list(box)


@pytest.mark.parametrize("n,graded", [((40, 22, 140), True), ((13, 11, 30), False), ((36, 9, 70), False)])
def test_interior_source_equals_oracle(n, graded):
    """The interior schedule: the split kernels outside the interior box and
    the one-pass kernel inside it (several tiles along every axis, feeder
    rows and quads inside and outside the box, x chunks starting inside it),
    old and new fields in two buffers: fields bit-exact with the oracle."""
    m = model(n, E.TRAPEZOIDAL, poles=False, graded=graded)
    state = random_state(m, seed=4)
    steps = 3
    got, box = run_interior(emu_lib(), m, state, steps)
    lo, hi = box[:3], box[3:]
    assert all(h > l for l, h in zip(lo, hi)) and lo[2] % 4 == 0 and hi[2] % 4 == 0
    want, _, _ = run_oracle(m, state, steps)
    for name, a, b in zip(["u_x", "u_y", "u_z", "i_x", "i_y", "i_z"], got, want):
        bad = np.argwhere(a.view(np.uint32) != b.view(np.uint32))
        assert bad.size == 0, f"{name}: {len(bad)} differ, first {tuple(bad[0])} (box {box})"


@pytest.mark.parametrize("n,graded,rows,planes", [
    ((13, 11, 30), False, 7, 5), ((20, 19, 140), True, 8, 32), ((9, 14, 131), False, 3, 4),
    ((17, 10, 7), True, 3, 3), ((14, 12, 36), False, 7, 4)])
def test_march_source_equals_oracle(n, graded, rows, planes):
    """The marching kernel (march.cuh): one pass of both updates and both
    CPML corrections over the whole grid, tensor-copied plane windows in a
    ring, recomputed rows below the tiles and nodes below the z tiles, x
    chunks, several z tiles (rows of 131 and 141 nodes) and row remainders,
    the layer nodes of each row corrected one per lane: fields bit-exact
    with the oracle. (The poles run after it in the pole kernel; the GPU
    tests cover them.)"""
    m = model(n, E.TRAPEZOIDAL, poles=False, graded=graded)
    state = random_state(m, seed=5)
    steps = 3
    arrs = [np.ascontiguousarray(x.copy()) for x in state]
    ptrs = (C.c_void_p * 6)(*[a.ctypes.data for a in arrs])
    lib = emu_lib()
    assert lib.emu_march_run(m.desc, steps, ptrs, rows, planes) == 0, lib.emu_error().decode()
    want, _, _ = run_oracle(m, state, steps)
    for name, a, b in zip(["u_x", "u_y", "u_z", "i_x", "i_y", "i_z"], arrs, want):
        bad = np.argwhere(a.view(np.uint32) != b.view(np.uint32))
        assert bad.size == 0, f"{name}: {len(bad)} differ, first {tuple(bad[0])}"


def test_march_bounded_wait_runs_out_and_reports():
    """The marching kernel's first block expects more bytes than its copies
    deliver: its wait gives up after the limit, the block sets the status
    flag and returns (every other block completes), so the step reports a
    timeout instead of hanging. A NaN in a field sets the divergence flag."""
    m = model((13, 11, 30), E.TRAPEZOIDAL, poles=False)
    lib = emu_lib()
    state = random_state(m, seed=6)
    arrs = [np.ascontiguousarray(x.copy()) for x in state]
    ptrs = (C.c_void_p * 6)(*[a.ctypes.data for a in arrs])
    assert lib.emu_march_timeout(m.desc, ptrs, 5_000_000) == 3, lib.emu_error().decode()
    arrs = [np.ascontiguousarray(x.copy()) for x in state]
    arrs[2][6, 5, 14] = np.nan
    ptrs = (C.c_void_p * 6)(*[a.ctypes.data for a in arrs])
    assert lib.emu_march_run(m.desc, 1, ptrs, 7, 4) == 4, lib.emu_error().decode()


def test_pole_capture_fold_decision():
    """The split schedule lets a pole kernel store the saved field values
    itself only when nothing between the correction and the reference's
    capture writes a pole edge: a source on a pole edge, or CPML applied after
    the dispersive hooks over a pole edge, keeps the capture kernel."""
    from helpers import mixed_model

    lib = emu_lib()
    m, _ = mixed_model(h_source=True)  # soft E source at the sphere's centre, soft H in the magnetic box
    assert lib.emu_pole_prev_fold(m.desc, 1) == 0
    assert lib.emu_pole_prev_fold(m.desc, 0) == 0
    m, _ = mixed_model(h_source=False)
    assert lib.emu_pole_prev_fold(m.desc, 1) == 0
    assert lib.emu_pole_prev_fold(m.desc, 0) == 1
    w = W.dispersive_box(n=40, radius=6, slab=3, cpml=4, steps=10)
    assert lib.emu_pole_prev_fold(w.model.desc, 1) == 1
    assert lib.emu_pole_prev_fold(w.model.desc, 0) == 0  # no magnetic poles
    # Dispersive medium registered before the CPML, its slab through the layers.
    m = E.Model.uniform([16, 16, 16], [1e-3] * 3)
    m.build()
    d = E.Dispersive()
    d.fill_cells(m, m.cells().box([0, 0, 6], [16, 16, 9]), [E.Pole.drude(6e10, 6e9)])
    m.add_dispersive(d, E.LEAPFROG)
    m.add_cpml([3] * 6)
    assert lib.emu_pole_prev_fold(m.desc, 1) == 0
    m = E.Model.uniform([16, 16, 16], [1e-3] * 3)
    m.build()
    d = E.Dispersive()
    d.fill_cells(m, m.cells().box([6, 6, 6], [9, 9, 9]), [E.Pole.drude(6e10, 6e9)])
    m.add_dispersive(d, E.LEAPFROG)
    m.add_cpml([3] * 6)
    assert lib.emu_pole_prev_fold(m.desc, 1) == 1


def test_fused_kernel_source_under_address_sanitizer():
    """The same emulation built with AddressSanitizer: no out-of-bounds access
    of any table, field, state or shared-memory buffer."""
    import shutil

    asan = subprocess.run(["gcc", "-print-file-name=libasan.so"], capture_output=True, text=True).stdout.strip()
    if not asan or not os.path.exists(asan):
        pytest.skip("libasan not available")
    code = (
        "import sys; sys.path[:0] = [%r, %r]\n"
        "import test_fused_emulation as T, ems_b200 as E\n"
        "m = T.model((11, 9, 14), E.LEAPFROG)\n"
        "T.run_emu(T.emu_lib(asan=True), m, T.random_state(m), 6, 4, 2)\n"
        "import ctypes as C, numpy as np\n"
        "m2 = T.model((9, 10, 13), E.TRAPEZOIDAL, magnetic=True)\n"
        "st = [np.ascontiguousarray(x) for x in T.random_state(m2)]\n"
        "p = (C.c_void_p * 6)(*[a.ctypes.data for a in st])\n"
        "assert T.emu_lib(asan=True).emu_two_run(m2.desc, 4, p, None) == 0\n"
        "m3 = T.model((10, 9, 12), E.TRAPEZOIDAL, poles=False)\n"
        "st = [np.ascontiguousarray(x) for x in T.random_state(m3)]\n"
        "p = (C.c_void_p * 6)(*[a.ctypes.data for a in st])\n"
        "assert T.emu_lib(asan=True).emu_split_run(m3.desc, 3, p, None) == 0\n"
        "m4 = T.model((36, 9, 70), E.TRAPEZOIDAL, poles=False)\n"
        "T.run_interior(T.emu_lib(asan=True), m4, T.random_state(m4), 2)\n"
        "print('clean')\n"
    ) % (HERE, os.path.dirname(HERE))
    env = dict(os.environ, LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0 and "clean" in r.stdout, r.stderr[-3000:]
