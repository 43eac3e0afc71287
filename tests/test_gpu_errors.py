"""Error paths of the CUDA engine that are tested without faulting a GPU.

* A bounded wait that runs out: the marching kernel's test hook arms one
  ring barrier with more expected bytes than its copies deliver (every copy
  lands; the phase never completes), its waits give up after 20 ms, the
  block sets the timeout flag and returns. The next check reports
  EMS_ERR_TIMEOUT; the handle and the context stay usable.
* Divergence: a NaN uploaded into a field makes the next marching step write
  non-finite values; the next check reports EMS_ERR_DIVERGED, and the run
  loop ends with the Diverged outcome (src/engine/run.rs:156-161).
"""
import numpy as np
import pytest

import ems_b200 as E
from ems_b200 import workloads as W
from oracle import OracleEngine
from helpers import assert_fields_equal

pytestmark = pytest.mark.gpu


def _box():
    return W.dispersive_box(n=40, radius=6, slab=3, cpml=4, steps=200)


def test_bounded_wait_runs_out_and_reports_timeout():
    w = _box()
    g = E.Engine(w.model)
    g.set_schedule(7)
    g.run(3)
    g.check()
    g.test_wait_timeout(20_000_000)
    g.run(1)
    with pytest.raises(E.EngineError) as ei:
        g.check()
    assert ei.value.status == E.ERR_TIMEOUT
    # The flag was cleared; the handle steps on.
    g.run(5)
    g.check()
    # The context is usable: a new engine on it matches the oracle.
    h = E.Engine(w.model)
    h.set_schedule(7)
    o = OracleEngine(w.model, threads=4)
    h.run(30)
    o.run(30)
    h.check()
    assert_fields_equal(h, o, "after a bounded wait ran out")


def test_nan_field_reports_divergence():
    w = _box()
    g = E.Engine(w.model)
    g.set_schedule(7)
    g.run(4)
    g.check()
    u = g.field(0, 2)
    u[20, 20, 20] = np.nan
    g.set_field(0, 2, u)
    g.run(2)
    with pytest.raises(E.EngineError) as ei:
        g.check()
    assert ei.value.status == E.ERR_DIVERGED


def test_run_loop_ends_diverged_on_nan():
    w = _box()
    g = E.Engine(w.model)
    g.set_schedule(7)
    g.run(10)
    u = g.field(1, 0)
    u[10, 12, 14] = np.inf
    g.set_field(1, 0, u)
    out = E.run_until(g, E.energy_decay_limits(2000, -40.0, w.model.dt))
    assert out.reason == 2  # Diverged
    assert out.checks == 1
