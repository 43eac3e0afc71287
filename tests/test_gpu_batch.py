"""Batches (ems_batch_*): many models stepping together equal each model run
alone, bit for bit, and the batched run loop equals the single one.

A batch is a sweep of uneven models; each must come out exactly as the
same model stepped alone by the engine (which the parity tests tie to the
oracle), whatever the other models in the launch, including a model frozen
mid-run."""
import numpy as np
import pytest

import ems_b200 as E
from ems_b200 import workloads as W
from helpers import assert_fields_equal, mixed_model, small_cavity

pytestmark = pytest.mark.gpu


class Alone:
    """A model of a batch, seen as an engine (field access for comparisons)."""

    def __init__(self, batch, m):
        self.b, self.m = batch, m

    def field(self, f, a):
        return self.b.field(self.m, f, a)


def _models():
    ws = [W.patch_variant(s, cells=(26, 44), steps=400) for s in (3, 4)]
    mixed, ops = mixed_model(scheme=E.LEAPFROG, steps=400)
    disp = W.dispersive_box(n=36, radius=5, slab=3, cpml=4, steps=400)
    cav, _ = small_cavity()
    models = [ws[0].model, mixed, disp.model, cav, ws[1].model]
    series = [[(ws[0].port, 0), (ws[0].port, 1), (ws[0].port, 2)],
              [(ops["pv"], 0), (ops["pi"], 0), (ops["pe"], 0), (ops["port"], 1), (ops["port"], 2)],
              [(p, 0) for p in disp.probes], [], [(ws[1].port, 1)]]
    return models, series


def test_batch_equals_each_model_alone():
    models, series = _models()
    b = E.Batch(models, max_steps=400)
    b.run(170)
    for q, m in enumerate(models):
        g = E.Engine(m)
        g.run(170)
        assert b.timestep(q) == 170
        assert_fields_equal(Alone(b, q), g, f"batch model {q}")
        for op, which in series[q]:
            x, y = b.samples(q, op, which), g.samples(op, which)
            assert x.shape == y.shape and x.size > 0
            assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), (q, op, which)


def test_batch_energy_and_freeze():
    models, _ = _models()
    b = E.Batch(models, max_steps=400)
    singles = [E.Engine(m) for m in models]
    for step in range(60):
        if step % 15 == 0:
            wb = b.step_with_energy()
            for q, g in enumerate(singles):
                if q == 2 and step >= 30:
                    assert wb[q] == 0.0  # frozen
                    continue
                wg = g.step_with_energy()
                assert abs(wb[q] - wg) <= 1e-12 * abs(wg), (q, wb[q], wg)
        else:
            b.run(1)
            for q, g in enumerate(singles):
                if not (q == 2 and step >= 30):
                    g.run(1)
        if step == 29:
            b.set_active(2, False)
    assert b.timestep(2) == 30 and b.timestep(0) == 60
    for q, g in enumerate(singles):
        assert_fields_equal(Alone(b, q), g, f"after freeze, model {q}")
    b.set_active(2, True)
    b.run(5)
    singles[2].run(5)
    assert_fields_equal(Alone(b, 2), singles[2], "resumed")


def test_batch_run_loop_equals_single_run_loops():
    """Lossy cavities of different conductivities stopping at −30 dB at
    different steps: the batched loop gives each the single loop's outcome."""
    kappas = [0.002, 0.004, 0.001]
    models = [small_cavity(kappa=k)[0] for k in kappas]
    t_end = small_cavity()[1]
    lims = [E.energy_decay_limits(20_000, -30.0, m.dt, excitation_end=t_end, interval=20) for m in models]
    want = [E.run_until(E.Engine(m), lim) for m, lim in zip(models, lims)]
    b = E.Batch(models, max_steps=20_000)
    got = E.run_until_batch(b, lims)
    for q, (g, w) in enumerate(zip(got, want)):
        assert (g.reason, g.steps, g.checks) == (w.reason, w.steps, w.checks), q
        assert g.energy == w.energy or abs(g.energy - w.energy) <= 1e-12 * abs(w.energy)
        assert b.timestep(q) == w.steps
    assert len({w.steps for w in want}) == 3  # the models stop at different steps


def test_batch_rejects_models_it_cannot_order():
    m = E.Model.uniform([10, 10, 10], [1e-3] * 3)
    m.build()
    m.add_probe(E.VOLTAGE, [(E.Z, (5, 5, 5), 1.0)])
    m.add_source(E.SOFT_E, [(E.Z, (4, 4, 4), 1.0)], 10e9, 5e9, 100)  # a probe before a source
    with pytest.raises(E.EngineError):
        E.Batch([m], max_steps=100)


def test_autotune_picks_and_caches_without_changing_results():
    import os

    cache = os.path.join(os.path.dirname(os.path.abspath(__file__)), ".cache", "autotune.txt")
    os.makedirs(os.path.dirname(cache), exist_ok=True)
    if os.path.exists(cache):
        os.remove(cache)
    m, _ = mixed_model(scheme=E.TRAPEZOIDAL, steps=60)
    g, ref = E.Engine(m), E.Engine(m)
    g.autotune(cache)
    g.run(40)  # 3 candidates × 4 steps tuned, the rest on the pick
    ref.run(40)
    assert_fields_equal(g, ref, "autotuned engine")
    lines = open(cache).read().splitlines()
    assert len(lines) == 1 and lines[0].startswith("engine ")
    pick = int(lines[0].split()[-2])
    assert g.schedule == pick
    h = E.Engine(m)
    h.autotune(cache)  # from the cache: no tuning steps
    assert h.schedule == pick
    models, _ = _models()
    b, singles = E.Batch(models, max_steps=100), [E.Engine(x) for x in models]
    b.autotune(cache)
    b.run(30)
    for q, x in enumerate(singles):
        x.run(30)
        assert_fields_equal(Alone(b, q), x, f"autotuned batch model {q}")
    assert any(l.startswith("batch ") for l in open(cache).read().splitlines())
