"""Shared helpers of the tests: small models and field comparison."""
from __future__ import annotations

import math

import numpy as np

import ems_b200 as E

TWO_PI = 2.0 * math.pi


def pulse(f0: float, bw: float):
    """The reference tests' Gaussian-modulated pulse (tests/engine.rs:15-23):
    τ = 1/(π·bw), centred at 4τ, over at 8τ. Returns (f, t_end)."""
    tau = 1.0 / (math.pi * bw)
    t0 = 4.0 * tau

    def f(t):
        x = (t - t0) / tau
        return np.exp(-x * x) * np.cos(2.0 * math.pi * f0 * (t - t0))

    return f, 2.0 * t0


def soft_e_table(f, dt: float, n_steps: int) -> np.ndarray:
    """Amplitudes of a soft E source for steps 0..n: f((n + ½)·dt)."""
    return np.array([f((s + 0.5) * dt) for s in range(n_steps)], dtype=np.float64)


def graded(length: float, cells: int, alpha: float) -> np.ndarray:
    """tests/engine.rs:72-82: sinusoidally graded lines."""
    t = np.arange(cells + 1) / cells
    return length * (t - alpha * np.sin(2.0 * math.pi * t) / (2.0 * math.pi))


def fields(eng) -> list[np.ndarray]:
    return [eng.field(f, a) for f in (0, 1) for a in (0, 1, 2)]


def assert_fields_equal(a, b, what: str = "") -> None:
    """Bit-exact comparison of the six field arrays of two engines."""
    names = ["u_x", "u_y", "u_z", "i_x", "i_y", "i_z"]
    fa, fb = fields(a), fields(b)
    # A comparison of all-zero fields would prove nothing.
    assert sum(int(np.count_nonzero(x)) for x in fa) > 0, f"{what}: fields are all zero"
    for name, x, y in zip(names, fa, fb):
        xb = x.view(np.uint32)
        yb = y.view(np.uint32)
        bad = np.count_nonzero(xb != yb)
        if bad:
            idx = np.argwhere(xb != yb)[0]
            raise AssertionError(f"{what} {name}: {bad} entries differ, first at {tuple(idx)}: "
                                 f"{x[tuple(idx)]!r} vs {y[tuple(idx)]!r}")


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    d = np.linalg.norm(np.asarray(a, dtype=np.float64) - np.asarray(b, dtype=np.float64))
    n = np.linalg.norm(np.asarray(b, dtype=np.float64))
    return float(d / n) if n > 0 else float(d)


def small_cavity(kappa: float = 0.0, threads_hint: int = 2):
    """tests/engine.rs:189-203: a 10×8×6 PEC cavity with two soft sources."""
    x = np.arange(11) * 0.01
    y = np.arange(9) * 0.009
    z = np.arange(7) * 0.011
    m = E.Model(x, y, z)
    if kappa:
        allc = m.cells().box([0, 0, 0], [10, 8, 6])
        m.fill(allc, m.material(kappa=kappa))
    m.build()
    f, t_end = pulse(3e9, 1e9)
    n_steps = int(math.ceil(t_end / m.dt)) + 4
    amp = soft_e_table(f, m.dt, n_steps)
    m.add_source_table(E.SOFT_E, [(E.Z, (3, 2, 2), 1.0), (E.X, (6, 5, 3), -0.5)], amp)
    return m, t_end


def mixed_model(n=(18, 16, 14), scheme=E.TRAPEZOIDAL, cpml=3, magnetic=True, lumped=True, steps=200, h_source=True):
    """A small model that exercises every operator: graded mesh, materials,
    a PEC box and a PMC face, CPML, electric Lorentz/Drude/Debye and
    magnetic poles, a lumped port, soft/hard E and H sources, voltage and
    current probes."""
    rng = np.random.default_rng(7)
    lines = [np.cumsum(np.concatenate([[0.0], 1e-3 * (1.0 + 0.2 * rng.random(c))])) for c in n]
    m = E.Model(*lines)
    diel = m.cells().box([3, 3, 3], [8, 9, 7])
    m.fill(diel, m.material(eps_r=(2.0, 3.0, 2.5), mu_r=1.2, kappa=0.01))
    m.fill_pec_box([11, 4, 4], [13, 7, 6])
    m.faces([E.PEC, E.PEC, E.PMC, E.PEC, E.PEC, E.PEC])
    m.build()
    ops = {}
    if cpml:
        ops["cpml"] = m.add_cpml([cpml, cpml, 0, cpml, cpml, cpml], kappa_max=2.0, alpha_max=0.05)
    d = E.Dispersive()
    d.fill_cells(m, m.cells().sphere([9.0, 8.0, 7.0], 3.5),
                 [E.Pole.lorentz(TWO_PI * 5e9, TWO_PI * 3e9, TWO_PI * 0.2e9),
                  E.Pole.lorentz(TWO_PI * 8e9, TWO_PI * 6e9, TWO_PI * 0.1e9)])
    d.fill_cells(m, m.cells().box([4, 10, 2], [14, 13, 5]), [E.Pole.drude(TWO_PI * 10e9, TWO_PI * 1e9)])
    d.fill_cells(m, m.cells().box([5, 2, 8], [9, 6, 11]), [E.Pole.debye(2.0, 20e-12)])
    if magnetic:
        d.fill_cells(m, m.cells().box([10, 9, 8], [14, 12, 11]), [E.Pole.lorentz(TWO_PI * 4e9, TWO_PI * 5e9, 1e8)],
                     field=1)
    ops["poles"] = m.add_dispersive(d, scheme)
    if lumped:
        ops["port"] = m.add_lumped_port(E.Z, [7, 11, 3], [7, 12, 5], 50.0, 4e9, 3e9, 1.0, steps)
    f, _ = pulse(6e9, 4e9)
    amp = soft_e_table(f, m.dt, steps)
    ops["soft_e"] = m.add_source_table(E.SOFT_E, [(E.Z, (9, 8, 7), 1.0), (E.Y, (6, 5, 9), -0.5)], amp)
    if h_source:
        ops["soft_h"] = m.add_source_table(E.SOFT_H, [(E.X, (12, 10, 9), 1e-3)], 0.5 * amp)
    ops["hard_e"] = m.add_source_table(E.HARD_E, [(E.X, (2, 2, 2), 1.0)], 0.1 * amp)
    ops["pv"] = m.add_probe(E.VOLTAGE, [(E.Z, (9, 8, 8), 1.0), (E.Z, (9, 8, 9), 1.0)])
    ops["pi"] = m.add_probe(E.CURRENT, [(E.X, (9, 8, 7), 1.0), (E.Y, (9, 8, 7), -1.0)], interval=3)
    ops["pe"] = m.add_probe(E.VOLTAGE, [(E.X, (5, 5, 5), 0.5)], interval=2)
    return m, ops
