"""Conducting sheets: the host's ladder set-up and the oracle's restatement of
the operator (src/engine/sheet.rs) against the reference's own tests.

* sheet.rs:1100-1148 (unit tests): the layer profile sums to the thickness
  and grades (48 layers for 35 µm of copper at 10 GHz, one for 35 nm at
  1 GHz); the exact slab's thin and thick limits; the ladder's face
  impedance Z11 within 1.2 % of the exact slab's from f_max/40 to f_max.
* tests/validation_sheet_conducting.rs:107-325, restated on the oracle:
  plane-wave transmission through a thin sheet (|T_meas/T_exact − 1| <
  2e-3) and a thick-ish one (< 0.35 dB and < 2° against the exact slab,
  < 5e-3 against the ladder model, while the thin-sheet formula is off by
  > 10 dB); the reflection loss 1 − |Γ| of a thick sheet (the one-sided
  surface resistance) within 3 %; a partial sheet in a closed cavity is
  passive and independent of the thread count; the energy invariant
  (nearly lossless: drift < 1e-5 over 2000 steps; lossy: non-increasing
  step by step) and an energy end criterion that fires at −4 dB.

The line is the quasi-1-D TEM line of tests/common/mod.rs:185-306 (one
5 mm cell across, PEC walls normal to E_x, PMC on the other pair, 8-cell
CPML at both ends), 0.25 mm cells. CPU only (the oracle).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import ems_b200 as E
from oracle import OracleEngine

Z0 = E.mu0() * E.c0()
TWO_PI = 2.0 * math.pi

DZ = 0.25e-3
CELLS, SRC, REFL, SHEET, TRANS = 480, 40, 140, 240, 400
STEPS = 2400
F_MAX = 15e9


# --------------------------------------------------------------------------
# sheet.rs unit tests (1100-1148).

def test_layer_profile_sums_and_grades():
    for s, t, f in [(5.8e7, 35e-6, 10e9), (5.8e7, 35e-9, 1e9), (1e5, 1e-3, 1e10)]:
        p = E.layer_profile(s, t, f)
        assert abs(p.sum() - t) < 1e-12 * t
        assert (p > 0.0).all()
    assert len(E.layer_profile(5.8e7, 35e-9, 1e9)) == 1
    assert len(E.layer_profile(5.8e7, 35e-6, 10e9)) == 48
    # The outer layers are 0.15 skin depths at f_max, growing by 1.15 inwards.
    p = E.layer_profile(5.8e7, 35e-6, 10e9)
    assert p[0] == pytest.approx(0.15 * E.skin_depth(5.8e7, 10e9), rel=1e-14)
    assert p[1] / p[0] == pytest.approx(1.15, rel=1e-12)
    assert np.array_equal(p, p[::-1])


def test_slab_thin_and_thick_limits():
    z11, z12 = E.slab_impedance(1e4, 1e-6, 1e9)
    r = 1.0 / (1e4 * 1e-6)
    assert abs(z11.real / r - 1.0) < 1e-3 and abs(z12.real / r - 1.0) < 1e-3
    s, f = 5.8e7, 10e9
    z11, z12 = E.slab_impedance(s, 1e-3, f)
    rs = 1.0 / (s * E.skin_depth(s, f))
    assert abs(z11 - complex(rs, rs)) < 1e-6 * rs
    assert abs(z12) < 1e-100


def test_ladder_matches_slab():
    for s, t, fmax in [(5.8e7, 35e-6, 10e9), (5.8e7, 1e-6, 10e9), (5.8e7, 5e-6, 10e9), (1e5, 1e-3, 10e9),
                       (1e3, 1e-4, 1e10)]:
        worst = 0.0
        for i in range(1, 41):
            f = fmax * i / 40.0
            m = E.model_abcd(s, t, fmax, f)
            x = E.slab_abcd(s, t, f)
            worst = max(worst, abs((m[0] / m[2]) / (x[0] / x[2]) - 1.0))
        assert worst < 0.012, (s, t, worst)


# --------------------------------------------------------------------------
# The line (tests/common/mod.rs:185-306, validation_sheet_conducting.rs:51-77).

def sine_pulse(f0, bw):
    tau = 1.0 / (math.pi * bw)
    t0 = 4.0 * tau
    return lambda t: math.exp(-((t - t0) / tau) ** 2) * math.sin(TWO_PI * f0 * (t - t0))


def line_model():
    z = np.arange(CELLS + 1) * DZ
    m = E.Model([0.0, 5e-3], [0.0, 5e-3], z)
    m.faces([E.PEC, E.PEC, E.PMC, E.PMC, E.PEC, E.PEC])
    return m


def run_line(kind):
    """kind None, "pec" or (sigma, t): (dt, series at REFL, series at TRANS)."""
    m = line_model()
    if kind == "pec":
        m.pec_edges(E.X, [0, 0, SHEET], [0, 1, SHEET])
    m.build()
    m.add_cpml([0, 0, 0, 0, 8, 8])
    f = sine_pulse(7e9, 4e9)
    amp = np.array([f((s + 0.5) * m.dt) for s in range(STEPS)])
    m.add_source_table(E.SOFT_E, [(E.X, (0, 0, SRC), 1.0), (E.X, (0, 1, SRC), 1.0)], amp)
    ps = [m.add_probe(E.VOLTAGE, [(E.X, (0, 0, k), 1.0)]) for k in (REFL, TRANS)]
    if isinstance(kind, tuple):
        sigma, t = kind
        op = m.add_sheet([(E.X, (0, j, SHEET), E.Z, sigma, t) for j in (0, 1)], f_max=F_MAX)
        assert m.sheet_edges[op] == (2, 0)
    o = OracleEngine(m, threads=1)
    o.run(STEPS)
    return m.dt, o.samples(ps[0]), o.samples(ps[1])


def spectrum(x, dt, freqs):
    return E.dft(dt, dt, np.asarray(x), freqs)


def freqs():
    return np.linspace(2e9, 12e9, 21)


def db(x):
    return 20.0 * math.log10(x)


def exact(sigma, t, f):
    a, b, c, d = E.slab_abcd(sigma, t, f)
    den = a + b / Z0 + c * Z0 + d
    return 2.0 / den, (a + b / Z0 - c * Z0 - d) / den


def transmission_of(m):
    a, b, c, d = m
    return 2.0 / (a + b / Z0 + c * Z0 + d)


@pytest.fixture(scope="module")
def vacuum():
    return run_line(None)


def transmission(ref, kind):
    dt, _, r = ref
    _, _, t = run_line(kind)
    f = freqs()
    return spectrum(t, dt, f) / spectrum(r, dt, f)


def test_thin_sheet_transmission(vacuum):
    """validation_sheet_conducting.rs:107-126: η0·σ·t = 3.77, T ≈ 0.347."""
    r = vacuum[2]
    assert np.abs(r[-50:]).max() / np.abs(r).max() < 1e-5
    sigma, t = 1e4, 1e-6
    tm = transmission(vacuum, (sigma, t))
    thin = 2.0 / (2.0 + Z0 * sigma * t)
    worst = 0.0
    for f, m in zip(freqs(), tm):
        te, _ = exact(sigma, t, f)
        assert abs((abs(te) - thin) / thin) < 1e-3
        worst = max(worst, abs(m / te - 1.0))
    assert worst < 2e-3, worst


def test_thick_sheet_transmission(vacuum):
    """validation_sheet_conducting.rs:128-166: σ = 1e6, t = 20 µm (1.8-4.4 δ)."""
    sigma, t = 1e6, 20e-6
    tm = transmission(vacuum, (sigma, t))
    thin = 2.0 / (2.0 + Z0 * sigma * t)
    worst = worst_phase = thin_off = worst_model = 0.0
    for f, m in zip(freqs(), tm):
        te, _ = exact(sigma, t, f)
        tl = transmission_of(E.model_abcd(sigma, t, F_MAX, f))
        worst = max(worst, abs(db(abs(m)) - db(abs(te))))
        worst_phase = max(worst_phase, abs(np.angle(m / te)))
        worst_model = max(worst_model, abs(m / tl - 1.0))
        thin_off = max(thin_off, abs(db(abs(te)) - db(thin)))
    assert thin_off > 10.0, thin_off
    assert worst < 0.35, worst
    assert math.degrees(worst_phase) < 2.0, worst_phase
    assert worst_model < 5e-3, worst_model


def test_thick_sheet_reflection_surface_resistance(vacuum):
    """validation_sheet_conducting.rs:168-197: σ = 1e4, t = 0.5 mm; the
    reflected wave against a PEC sheet's (Γ = −1)."""
    incident = vacuum[1]
    dt, pec, _ = run_line("pec")
    sigma, t = 1e4, 0.5e-3
    _, sheet, _ = run_line((sigma, t))
    f = freqs()
    rp = spectrum(pec - incident, dt, f)
    rs = spectrum(sheet - incident, dt, f)
    worst = 0.0
    for fq, a, b in zip(f, rp, rs):
        g = -b / a
        _, ge = exact(sigma, t, fq)
        worst = max(worst, abs((1.0 - abs(g)) / (1.0 - abs(ge)) - 1.0))
        assert abs(g / ge - 1.0) < 1e-3, (fq, g, ge)
    assert worst < 0.03, worst


# --------------------------------------------------------------------------
# The cavity (validation_sheet_conducting.rs:199-330).

def cavity_model(sigma, t):
    ys = [1e-3 * i ** 1.1 for i in range(13)]
    m = E.Model(np.linspace(0.0, 10e-3, 11), ys, np.linspace(0.0, 9e-3, 10))
    m.build()
    op = m.add_sheet_rect(E.Z, 4, [2, 3, 0], [8, 9, 0], sigma, t, f_max=20e9)
    return m, op


def seed_fields(o, m):
    for axis, node, v in ((E.Y, (3, 4, 2), 1.0), (E.X, (5, 6, 6), -0.7), (E.Z, (4, 5, 3), 0.4)):
        a = np.zeros(m.nodes, dtype=np.float32)
        a[node] = v
        o.set_field(0, axis, a)


def test_sheet_in_cavity_is_passive_and_deterministic():
    def run(threads, sigma, t):
        m, op = cavity_model(sigma, t)
        o = OracleEngine(m, threads=threads)
        seed_fields(o, m)
        w = [o.step_with_energy()]
        for _ in range(40):
            o.run(49)
            w.append(o.step_with_energy())
        return w, o.field(0, E.X), o.field(1, E.Y), m.sheet_edges[op]

    for sigma, t in [(1e4, 1e-6), (1e6, 20e-6), (5.8e7, 35e-6)]:
        w, ux, iy, (edges, skipped) = run(1, sigma, t)
        assert (edges, skipped) == (6 * 7 + 6 * 7, 0)
        w0 = w[0]
        for a, b in zip(w, w[1:]):
            assert b <= a * (1.0 + 1e-6) + 1e-12 * w0, (sigma, t, w)
        assert w[-1] < w0
        w4, ux4, iy4, _ = run(4, sigma, t)
        assert w == w4
        assert np.array_equal(ux, ux4) and np.array_equal(iy, iy4)


def test_sheet_energy_invariant():
    def build(sigma, t):
        m, _ = cavity_model(sigma, t)
        o = OracleEngine(m, threads=2)
        seed_fields(o, m)
        o.run(3)
        return m, o

    # Nearly lossless: conserved.
    _, o = build(1e-9, 1e-6)
    w = np.array([o.step_with_energy() for _ in range(2000)])
    assert (w.max() - w.min()) / w[0] < 1e-5
    # Lossy: non-increasing step by step.
    for sigma, t in [(1e4, 1e-6), (5.8e7, 35e-6)]:
        _, o = build(sigma, t)
        w = [o.step_with_energy() for _ in range(1000)]
        for a, b in zip(w, w[1:]):
            assert b <= a * (1.0 + 1e-6) + 1e-12 * w[0], (sigma, t)
    # The modes that miss the sheet hold the energy about 5 dB down: a −4 dB
    # criterion fires, at the reported level.
    m, o = build(1e4, 1e-6)
    w_start = o.step_with_energy()
    out = E.run_until(o, E.energy_decay_limits(20_000, -4.0, m.dt))
    w_end = o.step_with_energy()
    assert out.reason == 0
    assert out.ratio_db <= -4.0 and 10.0 * math.log10(w_end / w_start) < -3.5


def test_sheet_validation():
    m, _ = cavity_model(1e4, 1e-6)
    with pytest.raises(Exception):
        m.add_sheet([(E.Z, (1, 1, 4), E.Z, 1e4, 1e-6)])  # not tangential
    with pytest.raises(Exception):
        m.add_sheet([(E.X, (1, 1, 4), E.Z, 0.0, 1e-6)])
    with pytest.raises(Exception):
        m.add_sheet([(E.X, (1, 1, 4), E.Z, 1e4, -1.0)])
    with pytest.raises(Exception):
        m.add_sheet([(E.X, (10, 1, 4), E.Z, 1e4, 1e-6)])  # x node 10 has no x edge
    with pytest.raises(Exception):
        m.add_sheet([(E.X, (1, 1, 4), E.Z, 1e4, 1e-6, (1.5, 0.5))])
    with pytest.raises(Exception):
        m.add_sheet([(E.X, (1, 1, 4), E.Z, 1e4, 1e-6)], f_max=-1.0)
    # PEC edges (a face of the closed cavity) and duplicates are skipped.
    op = m.add_sheet([(E.X, (1, 0, 4), E.Z, 1e4, 1e-6), (E.X, (1, 1, 4), E.Z, 1e4, 1e-6),
                      (E.X, (1, 1, 4), E.Z, 1e4, 1e-6)])
    assert m.sheet_edges[op] == (1, 2)
