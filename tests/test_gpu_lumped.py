"""Lumped elements with branch state (inductors, series R + L + C) and ports
with their own source tables on the CUDA engine against the oracle: the
strip loop of the reference's lumped tests with a parallel RLC load and a
series RLC element, and the two-port with unequal port resistances, on
every schedule that runs lumped elements. Fields, port voltage and current
and the element's current record bit for bit; energies (branch energy
included) within 1e-12.
"""
import numpy as np
import pytest

import ems_b200 as E
from oracle import OracleEngine
from helpers import assert_fields_equal
from test_oracle_lumped import col, cube, gaussian_table, loop_model, LOAD_X, PORT_X

pytestmark = pytest.mark.gpu

ENERGY_RTOL = 1e-12
STEPS = 600


def _equal(a, b, what):
    assert a.shape == b.shape and a.size > 0, what
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), (what, np.max(np.abs(a - b)))


def _loop_with_branches():
    m = loop_model()
    amp = gaussian_table(0.0, 3e9, m.dt, STEPS)
    port = m.add_lumped_port_table(E.Z, *col(PORT_X), 50.0, amp)
    load = m.add_lumped(E.Z, *col(LOAD_X), r=200.0, l=8e-9, c=0.5e-12, record=True)
    ser = m.add_lumped(E.X, [9, 5, 10], [11, 5, 10], r=20.0, l=5e-9, c=2e-12, series=True, record=True,
                       amp=0.3 * amp)
    ind = m.add_lumped(E.Y, [14, 4, 7], [14, 6, 7], l=10e-9)
    return m, port, [load, ser, ind]


@pytest.mark.parametrize("schedule", [1, 3, 4, 5])
def test_branch_elements_bit_exact(schedule):
    m, port, els = _loop_with_branches()
    g = E.Engine(m)
    g.set_schedule(schedule)
    assert g.schedule == schedule
    o = OracleEngine(m, threads=2)
    eg, eo = [], []
    for s in range(0, STEPS, 40):
        eg.append(g.step_with_energy())
        eo.append(o.step_with_energy())
        g.run(39)
        o.run(39)
    assert_fields_equal(g, o, f"branch elements, schedule {schedule}")
    for which in (0, 1, 2):
        _equal(g.samples(port, which), o.samples(port, which), f"port {which}")
    for e in els[:2]:
        _equal(g.samples(e, 0), o.samples(e, 0), f"element {e} record")
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)


def test_two_port_bit_exact():
    m = cube(20)
    y, z0, z1 = 10, 9, 11
    for z in (z0, z1):
        m.fill_pec_box([5, y, z], [16, y + 1, z + 1])
    m.build()
    amp = gaussian_table(0.0, 3e9, m.dt, STEPS)
    p1 = m.add_lumped_port_table(E.Z, [5, y, z0], [5, y, z1], 50.0, amp)
    p2 = m.add_lumped_port_table(E.Z, [15, y, z0], [15, y, z1], 75.0, None)
    m.add_lumped(E.Z, [7, y, z0], [7, y, z1], c=0.5e-12)
    m.add_lumped(E.Z, [10, y, z0], [10, y, z1], r=30.0, c=2e-12, series=True)
    g = E.Engine(m)
    o = OracleEngine(m, threads=3)
    g.run(STEPS)
    o.run(STEPS)
    assert_fields_equal(g, o, "two-port")
    for p in (p1, p2):
        for which in (1, 2):
            _equal(g.samples(p, which), o.samples(p, which), f"port {p} {which}")
