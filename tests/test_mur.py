"""The Mur absorbing boundary: host set-up and the oracle against the
reference's own tests of it.

* entry counts, validation and the local cell size
  (src/engine/boundary/mur.rs:866-923);
* normal-incidence reflection of a TEM pulse below -30 dB on every axis,
  the PEC sanity check at 0 dB, energy leaving an all-Mur box, late-time
  stability and thread determinism (tests/mur.rs:1-246), on the oracle;
* the local-medium coefficient, the openEMS options and the held faces.

CPU only (the oracle and the host library); the CUDA engine's parity with
the oracle on these models is in test_gpu_parity.py.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import ems_b200 as E
from helpers import soft_e_table
from oracle import OracleEngine

C0 = E.c0()
D = 1e-3
TAU = 2.8e-11


def gaussian(t):
    """Gaussian of 1/e half-width TAU delayed by 4 TAU (tests/mur.rs:10-16)."""
    x = (t - 4.0 * TAU) / TAU
    return math.exp(-x * x)


def dgaussian(t):
    """Its derivative (tests/mur.rs:18-25)."""
    x = (t - 4.0 * TAU) / TAU
    return -2.0 * x * math.exp(-x * x)


def coefficient(v, dt, delta):
    """MurBoundary::coefficient (src/engine/boundary/mur.rs:725-727)."""
    return (v * dt - delta) / (v * dt + delta)


def uniform(cells, d=D):
    return [np.arange(c + 1) * d for c in cells]


NO_MUR = object()


def line_model(a, cells, src, probes, mur, steps, eps_r=1.0):
    """tests/mur.rs:30-86: a quasi-1-D line along a, one cell across, E
    along b = a+1, PEC on the b faces, PMC on the c = a+2 faces, Mur on both
    a faces unless `mur` is NO_MUR (True: C0, a number: that velocity, None:
    the local medium); a soft Gaussian source on plane src."""
    b, c = (a + 1) % 3, (a + 2) % 3
    n = [1, 1, 1]
    n[a] = cells
    m = E.Model(*uniform(n))
    faces = [E.PEC] * 6
    faces[2 * c] = faces[2 * c + 1] = E.PMC
    m.faces(faces)
    if eps_r != 1.0:
        m.fill(m.cells().box([0, 0, 0], n), m.material(eps_r=eps_r))
    m.build()
    if mur is not NO_MUR:
        v = C0 if mur is True else mur
        m.add_mur({2 * a: v, 2 * a + 1: v})

    def node(pos, q):
        p = [0, 0, 0]
        p[a] = pos
        p[c] = q
        return tuple(p)

    m.add_source_table(E.SOFT_E, [(b, node(src, 0), 1.0), (b, node(src, 1), 1.0)],
                       soft_e_table(gaussian, m.dt, steps))
    ks = [m.add_probe(E.VOLTAGE, [(b, node(p, 0), 1.0)]) for p in probes]
    return m, ks, node, b


def line(a, cells, src, probes, mur, steps, eps_r=1.0):
    m, ks, node, b = line_model(a, cells, src, probes, mur, steps, eps_r)
    o = OracleEngine(m, threads=1)
    o.run(steps)
    u = o.field(0, b)
    for p in probes:  # the exact TEM solution stays uniform across the line
        v0, v1 = float(u[node(p, 0)]), float(u[node(p, 1)])
        assert abs(v0 - v1) <= 1e-5 * max(abs(v0), 1e-6), (v0, v1)
    return [o.samples(k) for k in ks]


def window_steps():
    dt = 0.99 * D / (C0 * math.sqrt(3.0))
    return int(8.5e-10 / dt)


def reflection_db(a, mur=True, eps_r=1.0, steps=None):
    """tests/mur.rs:88-114: peak |Mur run - long reference line| over the
    incident peak, at both probes."""
    cells, src, probes, ext = 120, 60, [30, 90], 150
    steps = steps or window_steps()
    refr = line(a, cells + 2 * ext, src + ext, [p + ext for p in probes], NO_MUR, steps, eps_r)
    mur = line(a, cells, src, probes, mur, steps, eps_r)
    out = []
    for r, q in zip(refr, mur):
        peak = np.max(np.abs(r))
        assert peak > 0.0
        out.append(20.0 * math.log10(np.max(np.abs(r - q)) / peak))
    return out


@pytest.mark.parametrize("a", [0, 1, 2])
def test_normal_incidence_reflection(a):
    for db in reflection_db(a):
        assert db < -30.0, (a, db)


def test_reflection_much_better_than_pec():
    steps = window_steps()
    r = line(0, 420, 210, [180], NO_MUR, steps)[0]
    p = line(0, 120, 60, [30], NO_MUR, steps)[0]
    db = 20.0 * math.log10(np.max(np.abs(r - p)) / np.max(np.abs(r)))
    assert db > -1.0


def mur_box(cells, graded, flags=0, faces=None):
    """tests/mur.rs:145-172: a cells^3 box, Mur (C0) on all six faces, a
    dipole pulse in the middle."""
    def lines(s):
        t = np.arange(cells + 1) / cells
        w = 0.2 * np.sin(6.0 * t) / 6.0 if graded else 0.0
        return s * cells * (t + w)

    m = E.Model(lines(D), lines(1.1 * D), lines(0.9 * D)).build()
    m.add_mur(faces or {f: C0 for f in range(6)}, flags=flags)
    h = cells // 2
    steps = int((8.0 * TAU + 3.0e-10) / m.dt) + 4000
    amp = np.array([dgaussian((s + 0.5) * m.dt) for s in range(steps)])
    m.add_source_table(E.SOFT_E, [(E.Z, (h, h, h), 1.0), (E.X, (h - 2, h + 1, h), 0.3)], amp)
    return m


def drain(o, steps):
    peak = 0.0
    w = 0.0
    for _ in range(steps):
        w = o.step_with_energy()
        peak = max(peak, w)
    return peak, w


def test_energy_leaves_through_mur_faces():
    m = mur_box(16, graded=False)
    o = OracleEngine(m, threads=2)
    peak, end = drain(o, int((8.0 * TAU + 3.0e-10) / m.dt))
    assert end < 1e-2 * peak, (end, peak)


def test_long_run_stable():
    """tests/mur.rs:197-221 (3000 steps after the pulse has left)."""
    m = mur_box(12, graded=True)
    o = OracleEngine(m, threads=2)
    peak, w0 = drain(o, int((8.0 * TAU + 3.0e-10) / m.dt))
    wmax = 0.0
    for q in range(3000):
        w = o.step_with_energy()
        if q % 50 == 0:
            wmax = max(wmax, w)
    assert math.isfinite(w)
    assert w0 < 1e-9 * peak, (w0, peak)
    assert wmax < 1e-9 * peak, (w0, wmax)


def test_deterministic_across_threads():
    def run(threads):
        m = mur_box(10, graded=True)
        o = OracleEngine(m, threads=threads)
        assert o.threads == threads
        o.run(250)
        return [o.field(f, a).view(np.uint32).copy() for f in (0, 1) for a in range(3)]

    one = run(1)
    assert any(np.any(x != 0) for x in one)
    for t in (3, 4):
        for x, y in zip(one, run(t)):
            assert np.array_equal(x, y)


def test_counts_and_validation():
    """src/engine/boundary/mur.rs:866-893 on a 4x3x5-cell grid."""
    def model(faces=None):
        m = E.Model(*uniform([4, 3, 5]))
        if faces:
            m.faces(faces)
        return m.build()

    m = model()
    t = m.mur_table(m.add_mur({"x_min": 3e8}))
    assert len(t["axis"]) == 3 * 6 + 4 * 5 and t["n_edges"] == len(t["axis"])
    m = model()
    t = m.mur_table(m.add_mur({"x_min": 3e8, "z_min": 3e8}))
    assert len(t["axis"]) - t["n_edges"] == 3
    assert len(t["axis"]) == (3 * 6 + 4 * 5) + (4 * 4 + 5 * 3) - 3
    m = model()
    t = m.mur_table(m.add_mur({f: 3e8 for f in range(6)}))
    assert len(t["axis"]) - t["n_edges"] == 4 * (4 + 3 + 5)
    for bad in ({"x_min": 0.0}, {"x_min": float("nan")}, {"x_min": -1.0}):
        with pytest.raises(ValueError):
            model().add_mur(bad)
    pmc = [E.PEC] * 5 + [E.PMC]
    with pytest.raises(ValueError):
        model(pmc).add_mur({"z_max": 3e8})
    model(pmc).add_mur({"z_min": 3e8})
    thin = E.Model(*uniform([1, 3, 3])).build()
    with pytest.raises(ValueError):
        thin.add_mur({"x_min": 3e8})


def test_local_cell_size():
    """src/engine/boundary/mur.rs:895-915: the coefficient uses the boundary
    cell of its own face."""
    m = E.Model([0.0, 1e-3, 3e-3, 3.5e-3], [0.0, 1e-3], [0.0, 1e-3]).build()
    t = m.mur_table(m.add_mur({"x_min": 2e8, "x_max": 2e8}))
    assert t["n_edges"] == len(t["axis"]) == 2 * (2 + 2)
    for e in range(len(t["axis"])):
        delta, inner = (1e-3, 1) if t["node"][e][0] == 0 else (0.5e-3, 2)
        assert t["inner"][e][0][0] == inner
        assert t["k"][e][0] == np.float32(coefficient(2e8, m.dt, delta))


def test_corner_entries():
    """An edge on two Mur faces reads one neighbour along each face normal;
    its capacitance is the doubly-interior neighbour's over full first cells."""
    m = E.Model(*uniform([4, 3, 5])).build()
    t = m.mur_table(m.add_mur({"x_min": 3e8, "z_min": 3e8}, flags=E.MUR_COUNT_ENERGY))
    ne = t["n_edges"]
    for e in range(ne, len(t["axis"])):
        node, (i0, i1) = t["node"][e], t["inner"][e]
        assert t["axis"][e] == E.Y and node[0] == 0 and node[2] == 0
        assert tuple(i0) == (1, node[1], 0) and tuple(i1) == (0, node[1], 1)
    # Uniform vacuum: the doubly-interior neighbour's capacitance eps0·D²/D,
    # whose first cells are already full.
    for e in range(ne, len(t["axis"])):
        assert t["cap"][e] == pytest.approx(E.eps0() * D, rel=1e-6)


def test_local_medium_velocity():
    """with_faces_in: a face without a velocity takes each edge's local
    c0/sqrt(eps_r mu_r) (src/engine/boundary/mur.rs:487-510)."""
    m = E.Model(*uniform([6, 4, 4]))
    m.fill(m.cells().box([0, 0, 0], [6, 4, 4]), m.material(eps_r=4.0))
    m.build()
    t = m.mur_table(m.add_mur({"x_min": None, "x_max": C0}))
    for e in range(len(t["axis"])):
        if t["node"][e][0] == 0:
            assert t["k"][e][0] == np.float32(coefficient(C0 / 2.0, m.dt, D))
        else:
            assert t["k"][e][0] == np.float32(coefficient(C0, m.dt, D))


def test_local_medium_absorbs_in_dielectric():
    """In an eps_r = 4 line a locally tuned face reflects well under 1 %,
    a vacuum-tuned one tens of per cent (the reason for with_faces_in)."""
    steps = 2 * window_steps()
    local = reflection_db(0, mur=None, eps_r=4.0, steps=steps)
    vacuum = reflection_db(0, mur=C0, eps_r=4.0, steps=steps)
    assert max(local) < -30.0, local
    assert min(vacuum) > -12.0, vacuum


@pytest.mark.parametrize("flags", [0, E.MUR_OPENEMS_ORDER, E.MUR_OPENEMS_CORNERS,
                                   E.MUR_OPENEMS_ORDER | E.MUR_OPENEMS_CORNERS])
def test_update_rules(flags):
    """One step of every entry against the reference's expressions in f32
    (src/engine/boundary/mur.rs:252-299): face edges i + k(x - b) (openEMS
    order (i - k b) + k x), shared edges the mean of both (openEMS: i0 - k0 b)."""
    m = mur_box(8, graded=True, flags=flags)
    t = m.mur_table(len(m.ops) - 2)
    o = OracleEngine(m, threads=1)
    o.run(40)
    before = [o.field(0, a) for a in range(3)]
    o.run(1)
    after = [o.field(0, a) for a in range(3)]
    f32 = np.float32
    order = bool(flags & E.MUR_OPENEMS_ORDER)

    def one(i, k, x, b):
        return (f32(i) - f32(k) * f32(b)) + f32(k) * f32(x) if order else f32(i) + f32(k) * (f32(x) - f32(b))

    for e in range(len(t["axis"])):
        a, node, inner, k = t["axis"][e], tuple(t["node"][e]), t["inner"][e], t["k"][e]
        b = before[a][node]
        i0, x0 = before[a][tuple(inner[0])], after[a][tuple(inner[0])]
        if e < t["n_edges"]:
            want = one(i0, k[0], x0, b)
        elif flags & E.MUR_OPENEMS_CORNERS:
            want = f32(i0) - f32(k[0]) * f32(b)
        else:
            i1, x1 = before[a][tuple(inner[1])], after[a][tuple(inner[1])]
            want = f32(0.5) * (one(i0, k[0], x0, b) + one(i1, k[1], x1, b))
        assert after[a][node].view(np.uint32) == f32(want).view(np.uint32), (e, after[a][node], want)


def test_count_energy_adds_boundary_edges():
    """count_energy adds sum 1/2 C u^2 over the boundary edges' last values."""
    plain = OracleEngine(mur_box(10, graded=False), threads=1)
    counted = OracleEngine(mur_box(10, graded=False, flags=E.MUR_COUNT_ENERGY), threads=1)
    w0 = w1 = 0.0
    for _ in range(80):
        w0 = plain.step_with_energy()
        w1 = counted.step_with_energy()
    assert w1 > w0 > 0.0
    assert w1 - w0 < 0.5 * w0


def test_held_face_stays_zero():
    """hold_faces: the held face's edges keep their PEC zero before the
    given step and are updated from it on."""
    m = E.Model(*uniform([10, 10, 10])).build()
    m.add_mur({f: C0 for f in range(6)}, hold={"x_min": 40})
    m.add_source_table(E.SOFT_E, [(E.Z, (1, 5, 5), 1.0)],
                       np.array([dgaussian((s + 0.5) * m.dt) for s in range(200)]))
    o = OracleEngine(m, threads=1)
    o.run(40)
    assert not np.any(o.field(0, E.Z)[0]) and not np.any(o.field(0, E.Y)[0])
    assert np.any(o.field(0, E.Z)[1])
    o.run(5)
    assert np.any(o.field(0, E.Z)[0])
