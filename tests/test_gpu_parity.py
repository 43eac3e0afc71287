"""Parity of the CUDA engine with the oracle (the reference's step restated).

Every test builds one model, runs the CUDA engine (through the C ABI of
include/ems_gpu.h) and the oracle on the same tables, and requires:

* the six field arrays equal bit for bit (f32 bit patterns);
* probe, port voltage/current and lumped-current series equal bit for bit
  (both sum their entries in entry order);
* energies within 1e-12 relative (a reduction: the GPU sums in another order).

The reference engine itself is bit-identical across thread counts
(src/engine/mod.rs:64-79), so bit-exact agreement is the bar.
"""
import numpy as np
import pytest

import ems_b200 as E
from ems_b200 import workloads as W
from oracle import OracleEngine
from helpers import assert_fields_equal, mixed_model, small_cavity

pytestmark = pytest.mark.gpu

ENERGY_RTOL = 1e-12


def _lockstep(model, steps, energy_every=0, threads=4, schedule=0):
    g = E.Engine(model)
    g.set_schedule(schedule)
    o = OracleEngine(model, threads=threads)
    eg, eo = [], []
    s = 0
    while s < steps:
        if energy_every and s % energy_every == 0:
            eg.append(g.step_with_energy())
            eo.append(o.step_with_energy())
            s += 1
        else:
            n = min(steps - s, (energy_every - s % energy_every) if energy_every else steps)
            g.run(n)
            o.run(n)
            s += n
    return g, o, np.array(eg), np.array(eo)


def _series_equal(g, o, op, which=0):
    a, b = g.samples(op, which), o.samples(op, which)
    assert a.shape == b.shape and a.size > 0
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), (op, which, np.max(np.abs(a - b)))


def test_vacuum_pec_cavity_bit_exact():
    m, _ = small_cavity()
    g, o, eg, eo = _lockstep(m, 300, energy_every=25)
    assert_fields_equal(g, o, "cavity")
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)


def test_lossy_cavity_bit_exact():
    m, _ = small_cavity(kappa=0.002)
    g, o, eg, eo = _lockstep(m, 200, energy_every=10)
    assert_fields_equal(g, o, "lossy cavity")
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)


@pytest.mark.parametrize("scheme", [E.TRAPEZOIDAL, E.LEAPFROG])
@pytest.mark.parametrize("schedule", [1, 3, 4])
def test_every_operator_bit_exact(scheme, schedule):
    """Every operator at once (magnetic poles and an H source included), on
    the per-operator kernels (1), the two-kernel schedule (3) and the split
    schedule (4)."""
    m, ops = mixed_model(scheme=scheme, steps=240)
    g, o, eg, eo = _lockstep(m, 240, energy_every=20, schedule=schedule)
    assert g.schedule == schedule
    assert_fields_equal(g, o, f"mixed scheme {scheme} schedule {schedule}")
    for name in ("pv", "pi", "pe"):
        _series_equal(g, o, ops[name])
    for which in (0, 1, 2):
        _series_equal(g, o, ops["port"], which)
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)


@pytest.mark.parametrize("scheme", [E.TRAPEZOIDAL, E.LEAPFROG])
def test_fused_schedule_bit_exact(scheme):
    """Without magnetic poles and H sources the fused single-pass kernel
    runs; it must equal the separate kernels and the oracle bit for bit."""
    m, ops = mixed_model(scheme=scheme, magnetic=False, h_source=False, steps=240)
    g, o, eg, eo = _lockstep(m, 240, energy_every=20, schedule=2)
    assert g.schedule == 2
    assert_fields_equal(g, o, f"fused vs oracle, scheme {scheme}")
    for sch in (1, 3, 4):
        s = E.Engine(m)
        s.set_schedule(sch)
        assert s.schedule == sch
        s.run(240)
        assert_fields_equal(g, s, f"fused vs schedule {sch}, scheme {scheme}")
    for name in ("pv", "pi", "pe"):
        _series_equal(g, o, ops[name])
    for which in (0, 1, 2):
        _series_equal(g, o, ops["port"], which)
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)


def test_two_kernel_schedule_where_fused_cannot_run():
    m, _ = mixed_model(magnetic=True, steps=10)
    g = E.Engine(m)
    assert g.schedule == 4
    g.set_schedule(3)
    assert g.schedule == 3
    with pytest.raises(E.EngineError):
        g.set_schedule(2)
    with pytest.raises(E.EngineError):
        g.set_schedule(5)


def test_odd_sizes_and_tile_remainders():
    # nz = 33 + 1 nodes (a row pitch remainder), ny odd, CPML of 1 cell.
    m = E.Model.uniform([7, 5, 33], [1e-3, 1.2e-3, 0.9e-3])
    m.build(courant=0.9)
    m.add_cpml([1, 1, 1, 1, 1, 1])
    m.add_source(E.SOFT_E, [(E.Y, (3, 2, 16), 1.0)], 20e9, 15e9, 400)
    p = m.add_probe(E.VOLTAGE, [(E.Y, (3, 2, 20), 1.0)])
    g, o, eg, eo = _lockstep(m, 150, energy_every=7)
    assert_fields_equal(g, o, "odd")
    _series_equal(g, o, p)
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)


def test_vacuum_box_configuration_bit_exact():
    """The plain-method configuration in full: 100³ cells, CPML 8, 2000 steps,
    4 E_z probes; fields and probe series bit-exact."""
    w = W.vacuum_box()
    g, o, _, _ = _lockstep(w.model, w.steps, threads=0)
    assert g.schedule == 4
    for p in w.probes:
        _series_equal(g, o, p)
    assert_fields_equal(g, o, "vacuum box")


def test_dispersive_box_small_bit_exact():
    w = W.dispersive_box(n=48, radius=8, slab=4, cpml=5, steps=300)
    g, o, eg, eo = _lockstep(w.model, 300, energy_every=30)
    assert g.schedule == 4
    assert_fields_equal(g, o, "dispersive box")
    for p in w.probes:
        _series_equal(g, o, p)
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)


def test_patch_antenna_port_series_bit_exact():
    w = W.patch_antenna(scale=0.4, steps=600)
    g, o, _, _ = _lockstep(w.model, 600, threads=0)
    for which in (0, 1, 2):
        _series_equal(g, o, w.port, which)
    assert_fields_equal(g, o, "patch")


def test_field_upload_roundtrip_and_initial_state():
    m, _ = small_cavity()
    g = E.Engine(m)
    o = OracleEngine(m, threads=2)
    rng = np.random.default_rng(3)
    for f in (0, 1):
        for a in range(3):
            v = (rng.standard_normal(m.nodes) * 1e-3).astype(np.float32)
            g.set_field(f, a, v)
            o.set_field(f, a, v)
            assert np.array_equal(g.field(f, a), v)
    g.run(37)
    o.run(37)
    assert_fields_equal(g, o, "from a random state")


def test_invalid_tables_rejected():
    m, _ = small_cavity()
    lib = E.gpu_lib()
    import ctypes as C
    h = C.c_void_p()
    assert lib.ems_gpu_create(None, 0, C.byref(h)) == 1
    g = E.Engine(m)
    with pytest.raises(E.EngineError):
        g.samples(99)


@pytest.mark.parametrize("n", [40, 67])
@pytest.mark.parametrize("schedule", [2, 3, 4, 6, 7])
def test_dispersive_box_chunks_and_tiles(n, schedule):
    """Sizes whose rows, tiles and x chunks leave remainders."""
    w = W.dispersive_box(n=n, radius=n / 6, slab=3, cpml=4, steps=120)
    g, o, eg, eo = _lockstep(w.model, 120, energy_every=15, schedule=schedule)
    assert g.schedule == schedule
    assert_fields_equal(g, o, f"dispersive {n}")
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)


def _row_cpml_model(n, faces):
    m = E.Model.uniform([n, n + 3, n + 7], [0.5e-3] * 3)
    sph = m.cells().sphere([n / 2, n / 2, n / 2], n / 6)
    m.fill(sph, m.material(eps_r=2.0))
    m.build()
    m.add_cpml(faces)
    d = E.Dispersive()
    d.fill_cells(m, sph, W.lorentz_poles(3))
    m.add_dispersive(d, E.LEAPFROG)
    amp = np.array([np.exp(-(((s + 0.5) * m.dt - 30e-12) / 10e-12) ** 2) for s in range(200)])
    m.add_source_table(E.SOFT_E, [(E.X, (n // 3, n // 2, n // 2), 1.0), (E.Z, (n // 2, 2, n // 2), 0.5)], amp)
    return m


@pytest.mark.parametrize("n,faces", [(40, [4] * 6), (33, [4, 3, 0, 4, 5, 2]), (29, [1, 2, 3, 0, 1, 6])])
def test_split_row_cpml(n, faces):
    """The split schedule's row CPML (every slab's correction inside the
    updates' CPML variant, no shell kernel), with every face or some faces
    in a layer: fields bit for bit against the oracle, energy steps (which
    take the shells) within 1e-12."""
    m = _row_cpml_model(n, faces)
    g = E.Engine(m)
    g.set_row_cpml(True)
    assert g.row_cpml and g.schedule == 4
    o = OracleEngine(m, threads=4)
    eg, eo = [], []
    for s in range(150):
        if s % 25 == 0:
            eg.append(g.step_with_energy())
            eo.append(o.step_with_energy())
        else:
            g.run(1)
            o.run(1)
    assert_fields_equal(g, o, f"row CPML {n} {faces}")
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)
    g.set_row_cpml(False)
    assert not g.row_cpml


def test_row_cpml_refused_without_cpml_first():
    m = E.Model.uniform([20, 20, 20], [0.5e-3] * 3)
    m.build()
    d = E.Dispersive()
    d.fill_cells(m, m.cells().sphere([10, 10, 10], 4), W.lorentz_poles(3))
    m.add_dispersive(d, E.LEAPFROG)
    m.add_cpml([3] * 6)
    g = E.Engine(m)
    with pytest.raises(E.EngineError):
        g.set_row_cpml(True)


def test_split_saved_values_across_uploads_and_schedule_switches():
    """The split schedule's pole kernels store the saved field values
    themselves where that is exact; a field upload or a step on another
    schedule makes the next split step capture them again."""
    w = W.dispersive_box(n=40, radius=6, slab=3, cpml=4, steps=200)
    m = w.model
    g = E.Engine(m)
    o = OracleEngine(m, threads=4)
    assert g.schedule == 4
    rng = np.random.default_rng(5)
    for sch, n in ((4, 25), (1, 7), (4, 9), (3, 5), (4, 11)):
        g.set_schedule(sch)
        g.run(n)
        o.run(n)
        if sch == 4:
            v = (rng.standard_normal(m.nodes) * 1e-3).astype(np.float32)
            g.set_field(0, 0, v)
            o.set_field(0, 0, v)
    g.set_schedule(4)
    g.run(30)
    o.run(30)
    assert_fields_equal(g, o, "split with uploads and switches")
    for p in w.probes:
        _series_equal(g, o, p)


@pytest.mark.parametrize("order", [0, 1])
def test_interior_schedule_uploads_switches_and_probes(order):
    """The interior schedule (one-pass kernel over the interior box, split
    kernels around it, two field buffers): probe series and fields bit for
    bit through energy steps (split, in place), a field upload, switches to
    and from other schedules, in both curl orders; refused where a hook sits
    between the two updates."""
    w = W.dispersive_box(n=72, radius=10, slab=4, cpml=6, steps=260)
    m = w.model
    g = E.Engine(m)
    g.set_curl_order(order)
    o = OracleEngine(m, threads=4)
    o.set_curl_order(order)
    rng = np.random.default_rng(9)
    eg, eo = [], []
    for sch, n in ((6, 40), (4, 7), (6, 33), (1, 5), (6, 60)):
        g.set_schedule(sch)
        assert g.schedule == sch
        eg.append(g.step_with_energy())
        eo.append(o.step_with_energy())
        g.run(n)
        o.run(n)
        if sch == 6 and n == 33:
            v = (rng.standard_normal(m.nodes) * 1e-3).astype(np.float32)
            g.set_field(1, 2, v)
            o.set_field(1, 2, v)
    g.set_schedule(6)
    g.run(31)
    o.run(31)
    assert_fields_equal(g, o, f"interior schedule, curl order {order}")
    for p in w.probes:
        _series_equal(g, o, p)
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)
    mm, _ = mixed_model(scheme=E.LEAPFROG, h_source=True, steps=20)
    with pytest.raises(E.EngineError):
        E.Engine(mm).set_schedule(6)


@pytest.mark.parametrize("shape,planes", [(0, 32), (1, 7), (2, 5), (3, 64)])
@pytest.mark.parametrize("order", [0, 1])
def test_march_schedule_uploads_switches_and_probes(order, shape, planes):
    """The marching schedule (one pass of both updates and both CPML
    corrections over the whole grid, TMA-staged plane windows, two field
    buffers) in every tile shape: probe series and fields bit for bit through
    energy steps (split, in place), a field upload, switches to and from
    other schedules, in both curl orders; refused where a hook sits between
    the two updates."""
    w = W.dispersive_box(n=72, radius=10, slab=4, cpml=6, steps=260)
    m = w.model
    g = E.Engine(m)
    g.set_curl_order(order)
    g.set_march(shape, planes)
    o = OracleEngine(m, threads=4)
    o.set_curl_order(order)
    rng = np.random.default_rng(9)
    eg, eo = [], []
    for sch, n in ((7, 40), (4, 7), (7, 33), (6, 5), (7, 60), (1, 4)):
        g.set_schedule(sch)
        assert g.schedule == sch
        eg.append(g.step_with_energy())
        eo.append(o.step_with_energy())
        g.run(n)
        o.run(n)
        if sch == 7 and n == 33:
            v = (rng.standard_normal(m.nodes) * 1e-3).astype(np.float32)
            g.set_field(1, 2, v)
            o.set_field(1, 2, v)
    g.set_schedule(7)
    g.run(31)
    o.run(31)
    assert_fields_equal(g, o, f"marching schedule, curl order {order}, shape {shape}")
    for p in w.probes:
        _series_equal(g, o, p)
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)
    mm, _ = mixed_model(scheme=E.LEAPFROG, h_source=True, steps=20)
    with pytest.raises(E.EngineError):
        E.Engine(mm).set_schedule(7)


def test_march_schedule_odd_grid_without_layers():
    """No CPML, a z extent of 131 nodes (two z tiles, the second one of
    three nodes), rows that leave a short last tile, a PMC face and lossy
    media: the marching schedule equals the oracle bit for bit."""
    m = E.Model.uniform([23, 13, 130], [1e-3, 1.1e-3, 0.9e-3])
    m.fill(m.cells().box([3, 2, 10], [15, 9, 100]), m.material(eps_r=3.0, kappa=0.02))
    m.faces([E.PEC, E.PMC, E.PEC, E.PEC, E.PEC, E.PEC])
    m.build()
    m.add_source(E.SOFT_E, [(E.Y, (11, 6, 64), 1.0)], 20e9, 15e9, 300)
    p = m.add_probe(E.VOLTAGE, [(E.Y, (11, 6, 70), 1.0)])
    g, o, eg, eo = _lockstep(m, 160, energy_every=16, schedule=7)
    assert g.schedule == 7
    assert_fields_equal(g, o, "march, odd grid")
    _series_equal(g, o, p)
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)


@pytest.mark.parametrize("h_source", [True, False])
def test_split_magnetic_poles(h_source):
    """Magnetic poles on the split schedule, with (capture kernel) and
    without (saved values stored by the pole kernel) an H source on a pole
    edge."""
    m, ops = mixed_model(scheme=E.LEAPFROG, h_source=h_source, steps=160)
    g, o, eg, eo = _lockstep(m, 160, energy_every=16, schedule=4)
    assert g.schedule == 4
    assert_fields_equal(g, o, f"split, magnetic poles, H source {h_source}")
    for which in (0, 1, 2):
        _series_equal(g, o, ops["port"], which)
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)


def test_freq_dump_equals_the_dft_of_the_oracle_states():
    """Device frequency dumps (src/engine/dump.rs FreqDump, native values,
    state timing) against X(f) = Σ_m x(t_m)·e^{−j2πf·t_m}·K·dt over the
    oracle's states m = 0, K, 2K, … (E at m·dt, H at (m − ½)·dt), E = u/Δ,
    H = i/Δ*."""
    m, _ = small_cavity()
    freqs = [1.5e9, 3.0e9, 4.2e9]
    g = E.Engine(m)
    de = g.add_freq_dump(0, (1, 1, 1), (8, 6, 5), freqs, stride=(2, 1, 2), interval=1)
    dh = g.add_freq_dump(1, (0, 2, 0), (10, 2, 6), freqs, interval=3)
    o = OracleEngine(m, threads=2)
    steps = 90
    want_e = np.zeros((len(freqs), 4, 6, 3, 3), dtype=complex)
    want_h = np.zeros((len(freqs), 11, 1, 7, 3), dtype=complex)
    inv_e = [m.inv_edge_lengths(a) for a in range(3)]
    inv_h = [m.inv_edge_lengths(a, dual=True) for a in range(3)]
    ie, je, ke = np.arange(1, 9, 2), np.arange(1, 7), np.arange(1, 6, 2)
    for s in range(steps + 1):
        if s:
            o.run(1)
        u = [o.field(0, a)[np.ix_(ie, je, ke)] for a in range(3)]
        xe = np.stack([u[0] * inv_e[0][ie][:, None, None], u[1] * inv_e[1][je][None, :, None],
                       u[2] * inv_e[2][ke][None, None, :]], axis=-1)
        for q, f in enumerate(freqs):
            want_e[q] += xe * np.exp(-2j * np.pi * f * s * m.dt) * m.dt
        if s % 3 == 0:
            ih, jh, kh = np.arange(0, 11), np.array([2]), np.arange(0, 7)
            i_ = [o.field(1, a)[np.ix_(ih, jh, kh)] for a in range(3)]
            xh = np.stack([i_[0] * inv_h[0][ih][:, None, None], i_[1] * inv_h[1][jh][None, :, None],
                           i_[2] * inv_h[2][kh][None, None, :]], axis=-1)
            for q, f in enumerate(freqs):
                want_h[q] += xh * np.exp(-2j * np.pi * f * (s - 0.5) * m.dt) * 3 * m.dt
    g.run(steps)
    for q in range(len(freqs)):
        ge, gh = g.freq_dump(de, q), g.freq_dump(dh, q)
        assert np.abs(ge).max() > 0 and np.abs(gh).max() > 0
        assert np.abs(ge - want_e[q]).max() <= 1e-9 * np.abs(want_e[q]).max()
        assert np.abs(gh - want_h[q]).max() <= 1e-9 * np.abs(want_h[q]).max()


def test_time_dump_equals_the_oracle_states():
    """Device time-domain dumps (src/engine/dump.rs TimeDump, native values,
    state timing, every K states): E = u/Δ and H = i/Δ* of the oracle's
    states m = 0, K, 2K, ... bit for bit, with dumps added before the run
    and between runs, across buffer growth."""
    m, _ = small_cavity()
    g = E.Engine(m)
    de = g.add_time_dump(0, (1, 1, 1), (8, 6, 5), stride=(2, 1, 2), interval=2)
    o = OracleEngine(m, threads=2)
    inv_e = [m.inv_edge_lengths(a) for a in range(3)]
    inv_h = [m.inv_edge_lengths(a, dual=True) for a in range(3)]
    ie, je, ke = np.arange(1, 9, 2), np.arange(1, 7), np.arange(1, 6, 2)
    ih, jh, kh = np.arange(0, 11), np.array([2]), np.arange(0, 7)
    want_e, want_h = [], []
    steps = 300
    for s in range(steps + 1):
        if s:
            o.run(1)
        if s % 2 == 0:
            u = [o.field(0, a)[np.ix_(ie, je, ke)].astype(np.float64) for a in range(3)]
            want_e.append(np.stack([u[0] * inv_e[0][ie][:, None, None], u[1] * inv_e[1][je][None, :, None],
                                    u[2] * inv_e[2][ke][None, None, :]], axis=-1))
        if s >= 100 and s % 7 == 0:
            i_ = [o.field(1, a)[np.ix_(ih, jh, kh)].astype(np.float64) for a in range(3)]
            want_h.append((s, np.stack([i_[0] * inv_h[0][ih][:, None, None], i_[1] * inv_h[1][jh][None, :, None],
                                        i_[2] * inv_h[2][kh][None, None, :]], axis=-1)))
    g.run(100)
    dh = g.add_time_dump(1, (0, 2, 0), (10, 2, 6), interval=7)
    g.run(steps - 100)
    se, ve = g.time_dump(de)
    assert list(se) == list(range(0, steps + 1, 2))
    assert np.array_equal(ve.view(np.uint64), np.stack(want_e).view(np.uint64))
    sh, vh = g.time_dump(dh)
    assert list(sh) == [s for s, _ in want_h]
    assert np.array_equal(vh.view(np.uint64), np.stack([v for _, v in want_h]).view(np.uint64))
    assert np.abs(vh).max() > 0


@pytest.mark.parametrize("planes", [3, 7, 64])
def test_sweep_schedule_bit_exact(planes):
    """The sweep schedule (chunks of `planes` x-planes, each chunk's H
    update, hooks, E update and hooks in turn) on every operator but magnetic
    sources, against the oracle; chunk edges fall inside the CPML layers,
    the dispersive blocks and the port."""
    m, ops = mixed_model(scheme=E.LEAPFROG, h_source=False, steps=160)
    g = E.Engine(m)
    g.set_sweep_planes(planes)
    g.set_schedule(5)
    assert g.schedule == 5
    o = OracleEngine(m, threads=4)
    eg, eo = [], []
    for s in range(160):
        if s % 16 == 0:
            eg.append(g.step_with_energy())
            eo.append(o.step_with_energy())
        else:
            g.run(1)
            o.run(1)
    assert_fields_equal(g, o, f"sweep, {planes} planes")
    for name in ("pv", "pi", "pe"):
        _series_equal(g, o, ops[name])
    for which in (0, 1, 2):
        _series_equal(g, o, ops["port"], which)
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)


def test_sweep_schedule_dispersive_box_and_refusals():
    w = W.dispersive_box(n=40, radius=6, slab=3, cpml=4, steps=200)
    g = E.Engine(w.model)
    g.set_sweep_planes(5)
    g.set_schedule(5)
    o = OracleEngine(w.model, threads=4)
    g.run(90)
    o.run(90)
    assert_fields_equal(g, o, "sweep dispersive box")
    for p in w.probes:
        _series_equal(g, o, p)
    m, _ = mixed_model(h_source=True, steps=10)
    h = E.Engine(m)
    with pytest.raises(E.EngineError):
        h.set_schedule(5)  # magnetic sources
