"""Parity of the CUDA engine's Mur boundary with the oracle.

The all-Mur boxes and lines of tests/mur.rs, every option of the operator
(openEMS order and shared-edge rule, counted energy, held faces, the local
medium), and Mur faces beside CPML layers, dispersive media touching a Mur
face, a lumped port and sources, on every schedule: fields and probe series
bit for bit, energies within 1e-12 relative.
"""
import numpy as np
import pytest

import ems_b200 as E
from helpers import TWO_PI, assert_fields_equal, pulse, soft_e_table
from oracle import OracleEngine
from test_mur import C0, line_model, mur_box

pytestmark = pytest.mark.gpu

ENERGY_RTOL = 1e-12


def _lockstep(model, steps, schedule=0, energy_every=10, threads=3):
    g = E.Engine(model)
    g.set_schedule(schedule)
    o = OracleEngine(model, threads=threads)
    eg, eo = [], []
    for s in range(0, steps, energy_every):
        eg.append(g.step_with_energy())
        eo.append(o.step_with_energy())
        n = min(energy_every - 1, steps - s - 1)
        if n > 0:
            g.run(n)
            o.run(n)
    np.testing.assert_allclose(eg, eo, rtol=ENERGY_RTOL, atol=0)
    return g, o


@pytest.mark.parametrize("schedule", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("flags", [0, E.MUR_OPENEMS_ORDER | E.MUR_COUNT_ENERGY, E.MUR_OPENEMS_CORNERS])
def test_mur_box_bit_exact(schedule, flags):
    m = mur_box(14, graded=True, flags=flags)
    g, o = _lockstep(m, 160, schedule)
    assert g.schedule == schedule
    assert_fields_equal(g, o, f"Mur box, schedule {schedule}, flags {flags}")


@pytest.mark.parametrize("a", [0, 1, 2])
def test_mur_line_probes_bit_exact(a):
    m, ks, _, _ = line_model(a, 120, 60, [30, 90], True, 300)
    g, o = _lockstep(m, 300)
    assert_fields_equal(g, o, f"line {a}")
    for k in ks:
        x, y = g.samples(k), o.samples(k)
        assert x.size and np.array_equal(x.view(np.uint64), y.view(np.uint64))


def test_mur_held_faces_and_local_medium():
    rng = np.random.default_rng(3)
    lines = [np.cumsum(np.concatenate([[0.0], 1e-3 * (1.0 + 0.3 * rng.random(c))])) for c in (16, 13, 11)]
    m = E.Model(*lines)
    m.fill(m.cells().box([0, 0, 0], [16, 13, 5]), m.material(eps_r=3.0, mu_r=1.5))
    m.build()
    m.add_mur({"x_min": None, "x_max": C0, "y_min": None, "z_max": 0.8 * C0}, hold={"x_min": 30, "z_max": 55},
              flags=E.MUR_COUNT_ENERGY)
    f, _ = pulse(20e9, 15e9)
    amp = soft_e_table(f, m.dt, 200)
    m.add_source_table(E.SOFT_E, [(E.Z, (1, 6, 5), 1.0), (E.Y, (8, 6, 9), 0.7)], amp)
    g, o = _lockstep(m, 200, schedule=4)
    assert_fields_equal(g, o, "held faces, local medium")


@pytest.mark.parametrize("schedule", [1, 3, 4, 5])
def test_mur_with_cpml_dispersive_port(schedule):
    """Mur on the y and z faces, CPML on the x faces, a Drude slab touching
    the y_min face (its pole edges include Mur edges), a lumped port, soft
    and hard sources, probes."""
    rng = np.random.default_rng(11)
    lines = [np.cumsum(np.concatenate([[0.0], 1e-3 * (1.0 + 0.2 * rng.random(c))])) for c in (20, 15, 13)]
    m = E.Model(*lines)
    m.fill(m.cells().box([4, 4, 3], [10, 9, 8]), m.material(eps_r=2.5, kappa=0.01))
    m.build()
    ops = {"cpml": m.add_cpml([3, 3, 0, 0, 0, 0], kappa_max=2.0, alpha_max=0.05)}
    ops["mur"] = m.add_mur({"y_min": C0, "y_max": C0, "z_min": C0, "z_max": 0.9 * C0})
    d = E.Dispersive()
    d.fill_cells(m, m.cells().box([6, 0, 2], [14, 3, 10]), [E.Pole.drude(TWO_PI * 10e9, TWO_PI * 1e9)])
    ops["poles"] = m.add_dispersive(d, E.TRAPEZOIDAL)
    ops["port"] = m.add_lumped_port(E.Z, [9, 10, 4], [9, 11, 6], 50.0, 8e9, 6e9, 1.0, 220)
    f, _ = pulse(10e9, 8e9)
    amp = soft_e_table(f, m.dt, 220)
    ops["soft"] = m.add_source_table(E.SOFT_E, [(E.Z, (11, 7, 6), 1.0), (E.Y, (9, 1, 6), 0.5)], amp)
    ops["hard"] = m.add_source_table(E.HARD_E, [(E.X, (15, 12, 2), 1.0)], 0.2 * amp)
    ops["pv"] = m.add_probe(E.VOLTAGE, [(E.Z, (12, 7, 6), 1.0), (E.Y, (8, 0, 6), 1.0)])
    ops["pi"] = m.add_probe(E.CURRENT, [(E.X, (11, 7, 6), 1.0)], interval=2)
    g, o = _lockstep(m, 220, schedule)
    assert g.schedule == schedule
    assert_fields_equal(g, o, f"Mur + CPML + poles + port, schedule {schedule}")
    for name in ("pv", "pi"):
        x, y = g.samples(ops[name]), o.samples(ops[name])
        assert x.size and np.array_equal(x.view(np.uint64), y.view(np.uint64)), name
    for which in (0, 1, 2):
        x, y = g.samples(ops["port"], which), o.samples(ops["port"], which)
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), which


def test_mur_refused_by_batches():
    m = mur_box(8, graded=False)
    with pytest.raises(E.EngineError):
        E.Batch([m, m])
