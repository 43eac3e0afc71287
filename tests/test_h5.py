"""HDF5 dump and probe files (ems_b200/h5.py) in the layout of the
reference's src/io/h5.rs: the lookup3 checksum against its published test
vectors, the objects, attributes, shapes and values of dump and probe files
read back through the module's reader, every header checksum, and the probe
group names of the reference's own test (h5.rs `group_names`). The sampled
values come from the oracle. CPU only.
"""
from __future__ import annotations

import struct

import numpy as np
import pytest

import ems_b200 as E
from ems_b200 import h5
from oracle import OracleEngine


def test_lookup3_published_vectors():
    """Bob Jenkins' lookup3.c driver values of hashlittle."""
    assert h5.lookup3(b"") == 0xDEADBEEF
    assert h5.lookup3(b"Four score and seven years ago") == 0x17770551
    assert h5.lookup3(b"Four score and seven years ago", 1) == 0xCD628161
    # Every tail length of the last 12-byte block.
    seen = {h5.lookup3(bytes(range(n))) for n in range(1, 40)}
    assert len(seen) == 39


def test_group_names_of_the_reference_test():
    assert h5.group_name("port_ut1") == "port_ut1"
    assert h5.group_name("a/b c") == "a_b_c"
    assert h5.group_name("") == "_"
    assert h5.group_name("..") == "_.."
    assert h5.group_name("é.x-1") == "_.x-1"


def _model():
    m = E.Model(np.array([0.0, 1.0, 2.5, 4.5, 5.0, 6.0]) * 1e-3, np.array([0.0, 0.7, 1.9, 2.4, 3.6]) * 1e-3,
                np.array([0.0, 0.4, 1.0, 2.2, 3.0, 3.5, 4.0]) * 1e-3)
    m.build()
    return m


def _run(m, sampler, steps):
    o = OracleEngine(m, threads=1)
    rng = np.random.default_rng(3)
    for f in range(2):
        for a in range(3):
            o.set_field(f, a, (rng.standard_normal(m.nodes) * 1e-3).astype(np.float32))
    snaps = []
    for s in range(steps):
        o.run(1)
        snaps.append(o.sample(sampler))
    return snaps


@pytest.mark.parametrize("quantity,position", [(E.DUMP_E, E.NODES), (E.DUMP_H, E.CELL_CENTERS)])
def test_time_dump_file(quantity, position):
    """A time-domain dump: root attributes, /mesh, /step, /time and the
    [n, nx, ny, nz, 3] f32 field in C order, read back equal."""
    m = _model()
    s = E.Sampler(m, quantity, position)
    snaps = _run(m, s, 4)
    steps = np.arange(1, 5, dtype=np.uint64)
    times = [s.time(int(k), m.dt) for k in steps]
    b = h5.time_dump_bytes("Et0", 7, s, steps, times, np.stack(snaps))
    assert b[:8] == b"\x89HDF\r\n\x1a\n"
    d = h5.read(b)
    q = s.name
    assert d["attrs"] == {"format": "ems-dump", "version": 1, "name": "Et0", "id": 7, "quantity": q,
                          "domain": "time", "position": "nodes" if position == E.NODES else "cell_centers",
                          "unit": h5.quantity_unit(q, False)}
    assert d["attrs"]["version"].dtype == np.uint32 and d["attrs"]["id"].dtype == np.uint32
    for ax, name in enumerate("xyz"):
        np.testing.assert_array_equal(d["mesh"][name]["data"], s.coords[ax])
        assert d["mesh"][name]["attrs"] == {"unit": "m"}
    np.testing.assert_array_equal(d["step"]["data"], steps)
    assert d["step"]["data"].dtype == np.uint64
    np.testing.assert_array_equal(d["time"]["data"], times)
    assert d["time"]["attrs"] == {"unit": "s"}
    f = d[q]["data"]
    assert f.dtype == np.float32 and f.shape == (4, *s.dims, 3)
    np.testing.assert_array_equal(f, np.stack(snaps).astype(np.float32).reshape(4, *s.dims, 3))
    assert d[q]["attrs"] == {"unit": h5.quantity_unit(q, False)}
    assert set(d) == {"attrs", "mesh", "step", "time", q}


def test_freq_dump_file_and_large_contiguous_data():
    """A frequency-domain dump: the complex field as the {r, i} compound
    (read as complex128), /frequency, the samples attribute; a field over
    4 KiB is stored contiguously, a small one inside its header."""
    m = _model()
    s = E.Sampler(m, E.DUMP_E, E.NODES)
    rng = np.random.default_rng(8)
    freqs = [1e9, 2e9, 3.5e9]
    vals = rng.standard_normal((3, *s.dims, 3)) + 1j * rng.standard_normal((3, *s.dims, 3))
    assert vals.size * 16 > 4096
    b = h5.freq_dump_bytes("Ef", 2, s, freqs, vals, samples=120)
    d = h5.read(b)
    assert d["attrs"]["domain"] == "frequency" and d["attrs"]["samples"] == 120
    assert d["attrs"]["samples"].dtype == np.uint64 and d["attrs"]["unit"] == "V*s/m"
    np.testing.assert_array_equal(d["frequency"]["data"], freqs)
    assert d["frequency"]["attrs"] == {"unit": "Hz"}
    f = d["E"]["data"]
    assert f.dtype == np.complex128 and f.shape == (3, *s.dims, 3)
    np.testing.assert_array_equal(f, vals)
    # The small frequency list lives in its header (compact layout).
    small = h5.freq_dump_bytes("Ef", 2, ("H", "nodes", ([0.0], [0.0, 1.0], [2.0])), [1e9], np.ones((1, 1, 2, 1, 3)),
                               samples=1)
    assert h5.read(small)["H"]["data"].shape == (1, 1, 2, 1, 3)


def test_probe_file():
    """Probe groups with their attributes and datasets; a repeated name gets
    the probe id, then a counter; scalar and vector values; frequencies only
    where the probe has some."""
    t = np.arange(5) * 1e-12
    probes = [h5.ProbeSeries("port ut1", "voltage", 1, 0, 1e-12, t, np.sin(t * 1e11), [1e9, 2e9]),
              h5.ProbeSeries("port ut1", "current", 2, 1, 1e-12, t, np.cos(t * 1e11)),
              h5.ProbeSeries("port_ut1", "efield", 2, 2, 1e-12, t, np.arange(15.0).reshape(5, 3)),
              h5.ProbeSeries("h", "hfield", 9, 3, 1e-12, t, np.ones((5, 3)))]
    d = h5.read(h5.probes_bytes(probes))
    assert d["attrs"] == {"format": "ems-probes", "version": 1}
    assert set(d) == {"attrs", "port_ut1", "port_ut1_2", "port_ut1_2_2", "h"}
    g = d["port_ut1"]
    assert g["attrs"] == {"name": "port ut1", "kind": "voltage", "id": 1, "number": 0, "dt": 1e-12}
    np.testing.assert_array_equal(g["time"]["data"], t)
    np.testing.assert_array_equal(g["values"]["data"], np.sin(t * 1e11))
    assert g["values"]["attrs"] == {"unit": "V"}
    np.testing.assert_array_equal(g["frequencies"]["data"], [1e9, 2e9])
    assert "frequencies" not in d["port_ut1_2"]
    assert d["port_ut1_2"]["values"]["attrs"] == {"unit": "A"}
    assert d["port_ut1_2_2"]["values"]["data"].shape == (5, 3)
    assert d["h"]["values"]["attrs"] == {"unit": "A/m"}


def test_structure_and_checksums():
    """The superblock (version 2, 8-byte offsets and lengths, end of file at
    the file's size) and every object header carry lookup3 checksums the
    reader verifies: a flipped byte anywhere in a header or the superblock
    is refused."""
    b = bytearray(h5.time_dump_bytes("d", 0, ("E", "nodes", ([0.0, 1.0], [0.0], [0.0, 2.0])), [1], [1e-12],
                                      np.ones((1, 2, 1, 2, 3))))
    assert b[8:12] == bytes([2, 8, 8, 0])
    eof, root = struct.unpack_from("<QQ", b, 28)
    assert eof == len(b) and b[root:root + 4] == b"OHDR"
    headers = [i for i in range(len(b)) if b[i:i + 4] == b"OHDR"]
    assert len(headers) == 8  # root, mesh, x, y, z, step, time and the field E
    for at in (5, 20, headers[3] + 12):
        bad = bytearray(b)
        bad[at] ^= 0x40
        with pytest.raises(h5.H5FormatError):
            h5.read(bytes(bad))


def test_errors():
    with pytest.raises(ValueError):
        h5.time_dump_bytes("d", 0, ("E", "nodes", ([0.0], [0.0], [0.0])), [1, 2], [0.0], np.ones((2, 1, 1, 1, 3)))
    with pytest.raises(ValueError):
        h5.time_dump_bytes("d", 0, ("E", "nodes", ([0.0], [0.0], [0.0])), [1], [0.0], np.ones((2, 1, 1, 1, 3)))
    with pytest.raises(ValueError):
        h5.time_dump_bytes("d", 0, ("Q", "nodes", ([0.0], [0.0], [0.0])), [1], [0.0], np.ones((1, 1, 1, 1, 3)))
    with pytest.raises(ValueError):
        h5.probes_bytes([h5.ProbeSeries("p", "power", 0, 0, 1.0, [0.0], [0.0])])
