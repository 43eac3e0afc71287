"""The batched run loop (ems_batch_drive) against the single-model loop
(ems_drive, src/engine/run.rs:424-540 restated): each model of a batch gets
exactly the outcome it gets alone. Runs on the CPU with scripted energy
curves (no engine), as the reference's run-loop tests script theirs
(src/engine/run.rs:588-673)."""
import math

import numpy as np

import ems_b200 as E


class Curve:
    """A stepper whose energy invariant follows w(n): rises, then decays at
    `rate` per step, optionally turning NaN at step `nan_at`."""

    def __init__(self, peak_at, rate, nan_at=None, scale=1.0):
        self.n = 0
        self.peak_at, self.rate, self.nan_at, self.scale = peak_at, rate, nan_at, scale

    def w(self, n):
        if self.nan_at is not None and n >= self.nan_at:
            return float("nan")
        if n <= self.peak_at:
            return self.scale * (n + 1) / (self.peak_at + 1)
        return self.scale * math.exp(-self.rate * (n - self.peak_at))

    def run(self, k):
        self.n += k

    def step_with_energy(self):
        v = self.w(self.n)
        self.n += 1
        return v


class FakeBatch:
    """Curves stepping together; frozen ones do not advance."""

    def __init__(self, curves):
        self.curves = curves
        self.n = len(curves)
        self.active = [True] * self.n

    def run(self, k):
        for c, a in zip(self.curves, self.active):
            if a:
                c.run(k)

    def step_with_energy(self):
        out = np.zeros(self.n)
        for q, (c, a) in enumerate(zip(self.curves, self.active)):
            if a:
                out[q] = c.step_with_energy()
        return out

    def set_active(self, m, a):
        self.active[m] = a


def _curves():
    return [
        dict(peak_at=120, rate=0.01),               # decays to the criterion
        dict(peak_at=50, rate=0.002),               # slower decay
        dict(peak_at=300, rate=0.05, nan_at=900),   # decays before its NaN step
        dict(peak_at=200, rate=1e-5),               # hits its step limit
        dict(peak_at=10, rate=0.3, nan_at=30),      # diverges
        dict(peak_at=400, rate=0.02, scale=1e-3),   # excitation ends late
    ]


def _limits(dt):
    lims = []
    for q, (mx, db, exc) in enumerate([(5000, -30.0, 100 * dt), (5000, -40.0, 60 * dt), (5000, -20.0, 0.0),
                                       (777, -40.0, 10 * dt), (5000, -30.0, 0.0), (3000, -25.0, 900 * dt)]):
        lims.append(E.energy_decay_limits(mx, db, dt, excitation_end=exc, interval=20))
    return lims


def test_batch_drive_equals_single_drive():
    dt = 1e-12
    lims = _limits(dt)
    want = []
    for kw, lim in zip(_curves(), lims):
        want.append(E.run_until(Curve(**kw), lim))
    b = FakeBatch([Curve(**kw) for kw in _curves()])
    got = E.run_until_batch(b, lims)
    reasons = set()
    for q, (g, w) in enumerate(zip(got, want)):
        key = lambda o: (o.reason, o.steps, o.checks, o.energy if o.energy == o.energy else "nan",  # noqa: E731
                         o.max_energy, o.ratio_db)
        assert key(g) == key(w), (q, key(g), key(w))
        assert b.curves[q].n == w.steps  # the frozen model stopped where it would alone
        reasons.add(w.reason)
    assert reasons >= {0, 1, 2}  # decay, step limit and divergence all exercised
    assert not any(b.active)


def test_batch_drive_rejects_mixed_intervals():
    dt = 1e-12
    lims = [E.energy_decay_limits(100, -30.0, dt, interval=20), E.energy_decay_limits(100, -30.0, dt, interval=25)]
    b = FakeBatch([Curve(10, 0.1), Curve(10, 0.1)])
    try:
        E.run_until_batch(b, lims)
    except ValueError:
        return
    raise AssertionError("mixed check intervals accepted")
