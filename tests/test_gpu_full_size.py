"""Parity of the CUDA engine with the oracle on the benchmark configurations
at their full sizes.

* The 512³ dispersive box (CPML 10, two-pole Lorentz sphere of radius 80
  cells, Drude slab of 20 cells, soft E_x sheet, leapfrog poles): 100 steps
  on the engine's automatic schedule and on the oracle; the six field arrays
  and all five probe series bit for bit, energies within 1e-12.
* The patch antenna on its graded mesh (about 195 × 197 × 78 cells, FR-4
  slab, 50 Ω lumped port, CPML on five faces) run to −40 dB through the run
  loop (src/engine/run.rs:424-540) on both: the same stop step, reason and
  number of checks, the port's voltage and current series bit for bit, and
  Z_in and S11 over 1–3 GHz (src/engine/port.rs:191-205,
  src/post/port.rs:202-209) within 1e-4 relative.

The oracle takes most of the time (about 0.2 s per step of the 512³ box and
a few ms per step of the patch on 16 host threads).
"""
import numpy as np
import pytest

import ems_b200 as E
from ems_b200 import workloads as W
from oracle import OracleEngine
from helpers import assert_fields_equal

pytestmark = pytest.mark.gpu

ENERGY_RTOL = 1e-12
PORT_RTOL = 1e-4


def _series_equal(g, o, op, which=0):
    a, b = g.samples(op, which), o.samples(op, which)
    assert a.shape == b.shape and a.size > 0
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), (op, which, np.max(np.abs(a - b)))


def test_dispersive_box_512_bit_exact():
    """The automatic schedule and the split schedule, each against the oracle."""
    w = W.dispersive_box(steps=120)
    assert w.cells == 512 ** 3
    gs = [E.Engine(w.model), E.Engine(w.model)]
    gs[1].set_schedule(4)
    o = OracleEngine(w.model, threads=0)
    eg, eo = [[], []], []
    for n in (1, 49, 1, 49):  # 100 steps, two of them with the energy invariant
        if n == 1:
            for q, g in enumerate(gs):
                eg[q].append(g.step_with_energy())
            eo.append(o.step_with_energy())
        else:
            for g in gs:
                g.run(n)
            o.run(n)
    for q, g in enumerate(gs):
        assert g.timestep == 100
        assert_fields_equal(g, o, f"512^3 dispersive box, schedule {g.schedule}")
        for p in w.probes:
            _series_equal(g, o, p)
        assert eg[q][-1] > 0.0
        np.testing.assert_allclose(eg[q], eo, rtol=ENERGY_RTOL, atol=0)


class _Counted:
    """A stepper that records how the run loop drove it."""

    def __init__(self, eng):
        self.eng = eng
        self.energies = []

    def run(self, n):
        self.eng.run(n)

    def step_with_energy(self):
        w = self.eng.step_with_energy()
        self.energies.append(w)
        return w


def test_patch_antenna_full_size_to_minus_40_db():
    w = W.patch_antenna(scale=1.0, steps=200_000)
    m = w.model
    assert 2.5e6 < w.cells < 3.5e6
    limits = E.energy_decay_limits(200_000, -40.0, m.dt, excitation_end=E.waveform_duration(2e9, 1e9))
    g, o = _Counted(E.Engine(m)), _Counted(OracleEngine(m, threads=0))
    out_g = E.run_until(g, limits)
    out_o = E.run_until(o, limits)
    assert out_g.reason == 0 and out_o.reason == 0  # stopped on the energy decay
    assert (out_g.steps, out_g.checks) == (out_o.steps, out_o.checks)
    assert out_g.ratio_db <= -40.0
    np.testing.assert_allclose(g.energies, o.energies, rtol=ENERGY_RTOL, atol=0)
    for which in (0, 1, 2):
        _series_equal(g.eng, o.eng, w.port, which)
    freqs = np.linspace(1e9, 3e9, 41)
    # Series 1 is the port voltage, 2 its current.
    zg, sg = E.port_result(g.eng.samples(w.port, 1), g.eng.samples(w.port, 2), m.dt, freqs)
    zo, so = E.port_result(o.eng.samples(w.port, 1), o.eng.samples(w.port, 2), m.dt, freqs)
    assert np.all(np.abs(zg - zo) <= PORT_RTOL * np.abs(zo))
    assert np.all(np.abs(sg - so) <= PORT_RTOL * np.abs(so))
    # The patch resonates in the band: |S11| dips below −3 dB.
    assert 20 * np.log10(np.abs(so)).min() < -3.0
