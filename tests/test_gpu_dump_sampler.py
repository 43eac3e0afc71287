"""Interpolated and derived field dumps on the CUDA engine (FieldSampler
tables, src/engine/dump.rs:487-940) against the oracle's sampling of the
same states: every quantity (E, H, J, rot H, D, B) at nodes, cell centres
and native positions, sub-sampled boxes, a degenerate cell-centre plane and
openEMS's explicit-index rules; time-domain snapshots bit for bit (f64),
the running DFT within 1e-9 of a DFT of the oracle's samples.
"""
import numpy as np
import pytest

import ems_b200 as E
from oracle import OracleEngine
from helpers import small_cavity

pytestmark = pytest.mark.gpu


def _samplers(m):
    n = m.nodes
    return [
        E.Sampler(m, E.DUMP_E, E.NODES),
        E.Sampler(m, E.DUMP_H, E.CELL_CENTERS),
        E.Sampler(m, E.DUMP_J, E.NATIVE, [1, 1, 1], [n[0] - 2, n[1] - 2, n[2] - 2], stride=[2, 1, 3]),
        E.Sampler(m, E.DUMP_ROTH, E.NODES, [0, 2, 0], [n[0] - 1, 2, n[2] - 1]),
        E.Sampler(m, E.DUMP_D, E.CELL_CENTERS, [n[0] - 1, 3, 0], [0, 3, n[2] - 1]),
        E.Sampler(m, E.DUMP_B, E.NODES, stride=[3, 2, 1]),
        E.Sampler(m, E.DUMP_H, E.NODES, indices=[range(0, n[0], 2), [1, 3, 4], range(n[2])]),
        E.Sampler(m, E.DUMP_ROTH, E.CELL_CENTERS, indices=[range(n[0]), [0, n[1] - 1], [2, 5]]),
    ]


def test_sampled_time_dumps_bit_exact():
    m, _ = small_cavity(kappa=0.02)
    ss = _samplers(m)
    g = E.Engine(m)
    ids = [g.add_sampled_time_dump(s, interval=5) for s in ss]
    o = OracleEngine(m, threads=2)
    want = [[] for _ in ss]
    steps = 120
    for s in range(steps + 1):
        if s:
            o.run(1)
        if s % 5 == 0:
            for q, sp in enumerate(ss):
                want[q].append(o.sample(sp))
    g.run(steps)
    for q, (sp, d) in enumerate(zip(ss, ids)):
        st, v = g.time_dump(d)
        assert list(st) == list(range(0, steps + 1, 5))
        w = np.stack(want[q]).reshape(v.shape)
        assert np.abs(w).max() > 0, (q, sp.name)
        assert np.array_equal(v.view(np.uint64), w.view(np.uint64)), (q, sp.name, np.abs(v - w).max())


def test_sampled_freq_dumps():
    m, _ = small_cavity(kappa=0.02)
    ss = _samplers(m)[:6]
    freqs = [1.5e9, 3.0e9, 4.2e9]
    g = E.Engine(m)
    ids = [g.add_sampled_freq_dump(s, freqs, interval=2) for s in ss]
    o = OracleEngine(m, threads=2)
    steps = 90
    want = [np.zeros((len(freqs), len(s), 3), dtype=complex) for s in ss]
    for s in range(steps + 1):
        if s:
            o.run(1)
        if s % 2:
            continue
        for q, sp in enumerate(ss):
            x = o.sample(sp)
            t = sp.time(s, m.dt)
            for k, f in enumerate(freqs):
                want[q][k] += x * np.exp(-2j * np.pi * f * t) * 2 * m.dt
    g.run(steps)
    for q, (sp, d) in enumerate(zip(ss, ids)):
        for k in range(len(freqs)):
            got = g.freq_dump(d, k).reshape(len(sp), 3)
            w = want[q][k]
            assert np.abs(w).max() > 0, (q, sp.name)
            assert np.abs(got - w).max() <= 1e-9 * np.abs(w).max(), (q, sp.name, k)


def test_dump_files_from_the_device(tmp_path):
    """The device dumps written as the reference's HDF5 dump files
    (ems_b200/h5.py) and read back: the snapshots as f32 of the device's
    values with their steps and times, the transform's complex values and
    the number of accumulated states."""
    from ems_b200 import h5

    m, _ = small_cavity(kappa=0.02)
    s_e = E.Sampler(m, E.DUMP_E, E.NODES)
    s_h = E.Sampler(m, E.DUMP_H, E.CELL_CENTERS)
    freqs = [2e9, 3e9]
    g = E.Engine(m)
    td = g.add_sampled_time_dump(s_h, interval=10)
    fd = g.add_sampled_freq_dump(s_e, freqs, interval=3)
    steps = 60
    g.run(steps)
    st, v = g.time_dump(td)
    h5.write_time_dump(str(tmp_path / "ht.h5"), "ht", 4, s_h, st, [s_h.time(int(k), m.dt) for k in st], v)
    d = h5.read(str(tmp_path / "ht.h5"))
    assert d["attrs"]["quantity"] == "H" and d["attrs"]["position"] == "cell_centers"
    np.testing.assert_array_equal(d["step"]["data"], st)
    np.testing.assert_array_equal(d["time"]["data"], [(k - 0.5) * m.dt for k in st])
    assert np.array_equal(d["H"]["data"], v.astype(np.float32)) and np.abs(v).max() > 0
    vals = np.stack([g.freq_dump(fd, k) for k in range(len(freqs))])
    h5.write_freq_dump(str(tmp_path / "ef.h5"), "ef", 5, s_e, freqs, vals, samples=steps // 3 + 1)
    d = h5.read(str(tmp_path / "ef.h5"))
    assert d["attrs"]["samples"] == steps // 3 + 1
    assert np.array_equal(d["E"]["data"], vals) and np.abs(vals).max() > 0
