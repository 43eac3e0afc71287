"""Conducting sheets on the CUDA engine against the oracle (src/engine/sheet.rs):
the partial sheet across the graded cavity of the reference's validation
tests (three conductivities, thin to thick against the skin depth), two
crossing sheets of different normals whose corrections meet on shared dual
edges, a sheet inside a CPML layer, and the transmission line with a sheet
across it. Fields, probe series and the ladders' voltages and currents bit
for bit; energies (ladder energy and H-correction term included) within
1e-12. Schedules that cannot run a serial hook between the H and E updates
refuse sheets.
"""
import numpy as np
import pytest

import ems_b200 as E
from oracle import OracleEngine
from helpers import assert_fields_equal
from test_oracle_sheet import cavity_model, run_line, seed_fields, line_model, SHEET, F_MAX

pytestmark = pytest.mark.gpu

ENERGY_RTOL = 1e-12


def _equal(a, b, what):
    assert a.shape == b.shape and a.size > 0, what
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), (what, np.max(np.abs(a - b)))


def _compare(m, ops, steps, schedule, threads=2):
    g = E.Engine(m)
    g.set_schedule(schedule)
    o = OracleEngine(m, threads=threads)
    seed_fields(g, m)
    seed_fields(o, m)
    eg, eo = [], []
    for _ in range(0, steps, 25):
        eg.append(g.step_with_energy())
        eo.append(o.step_with_energy())
        g.run(24)
        o.run(24)
    assert_fields_equal(g, o, f"sheets, schedule {schedule}")
    for op in ops:
        for which in (0, 1):
            _equal(g.samples(op, which), o.samples(op, which), f"sheet {op} ladder {which}")
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)
    return g


@pytest.mark.parametrize("schedule", [0, 1, 3, 4])
@pytest.mark.parametrize("sigma,t", [(1e4, 1e-6), (1e6, 20e-6), (5.8e7, 35e-6)])
def test_cavity_sheet_bit_exact(schedule, sigma, t):
    m, op = cavity_model(sigma, t)
    g = _compare(m, [op], 400, schedule)
    assert g.schedule in (1, 3, 4)


def test_crossing_sheets_share_dual_edges():
    """A z-normal and an x-normal sheet meeting along a line, and a second
    z-normal op over part of the first: dual edges get corrections from
    several edges and ops, which must apply in the reference's order."""
    ys = [1e-3 * i ** 1.1 for i in range(13)]
    m = E.Model(np.linspace(0.0, 10e-3, 11), ys, np.linspace(0.0, 9e-3, 10))
    m.build()
    a = m.add_sheet_rect(E.Z, 4, [2, 3, 0], [8, 9, 0], 1e6, 20e-6, f_max=20e9)
    b = m.add_sheet_rect(E.X, 5, [0, 2, 2], [0, 10, 7], 5.8e7, 35e-6, f_max=20e9)
    c = m.add_sheet(E.sheet_rect_edges(E.Z, 6, [1, 1, 0], [4, 5, 0], 1e4, 1e-6)
                    + [(E.X, (6, 6, 6), E.Z, 1e5, 5e-6, (0.3, 0.7))], f_max=15e9)
    for schedule in (1, 4):
        _compare(m, [a, b, c], 300, schedule, threads=3)


def test_sheet_in_cpml_layer():
    """Sheet edges inside a CPML lose its correction (the operator rewrites
    them after the slab hooks), on both engines alike."""
    m = E.Model.uniform([14, 14, 14], [1e-3] * 3)
    m.build()
    m.add_cpml([4, 4, 4, 4, 4, 4])
    op = m.add_sheet_rect(E.Z, 7, [1, 1, 0], [12, 12, 0], 1e5, 5e-6, f_max=30e9)
    amp = np.array([np.exp(-(((s + 0.5) * m.dt - 40e-12) / 12e-12) ** 2) for s in range(400)])
    m.add_source_table(E.SOFT_E, [(E.X, (6, 7, 3), 1.0)], amp)
    pr = m.add_probe(E.VOLTAGE, [(E.X, (6, 7, 11), 1.0)])
    for schedule in (1, 3, 4):
        g = E.Engine(m)
        g.set_schedule(schedule)
        o = OracleEngine(m, threads=2)
        g.run(400)
        o.run(400)
        assert_fields_equal(g, o, f"sheet in CPML, schedule {schedule}")
        _equal(g.samples(pr), o.samples(pr), "probe")
        _equal(g.samples(op, 0), o.samples(op, 0), "ladder u")


def test_line_with_sheet_bit_exact():
    """The transmission line of the reference's sheet validation, thick-ish
    sheet: both probe series bit for bit over the whole 2400-step record."""
    dt, refl, trans = run_line((1e6, 20e-6))
    m = line_model()
    m.build()
    m.add_cpml([0, 0, 0, 0, 8, 8])
    from test_oracle_sheet import sine_pulse, SRC, REFL, TRANS, STEPS
    f = sine_pulse(7e9, 4e9)
    amp = np.array([f((s + 0.5) * m.dt) for s in range(STEPS)])
    m.add_source_table(E.SOFT_E, [(E.X, (0, 0, SRC), 1.0), (E.X, (0, 1, SRC), 1.0)], amp)
    ps = [m.add_probe(E.VOLTAGE, [(E.X, (0, 0, k), 1.0)]) for k in (REFL, TRANS)]
    m.add_sheet([(E.X, (0, j, SHEET), E.Z, 1e6, 20e-6) for j in (0, 1)], f_max=F_MAX)
    g = E.Engine(m)
    g.run(STEPS)
    _equal(g.samples(ps[0]), refl, "reflection probe")
    _equal(g.samples(ps[1]), trans, "transmission probe")


def test_schedules_without_serial_post_h_refuse_sheets():
    m, _ = cavity_model(1e6, 20e-6)
    g = E.Engine(m)
    for s in (2, 5, 6, 7):
        with pytest.raises(E.EngineError):
            g.set_schedule(s)
    with pytest.raises(E.EngineError):
        E.Batch([m])
