"""The VTK writers (ems_b200/vtr.py) against the reference's writer tests
(src/io/vtr/tests.rs:199-520) and its dump-file test (tests/dump.rs:444-489),
with dumps sampled on the oracle. CPU only.
"""
from __future__ import annotations

import base64
import os
import re
import struct

import numpy as np
import pytest

import ems_b200 as E
from ems_b200 import vtr as V
from oracle import OracleEngine
from test_oracle_dump import analytic_model, set_analytic

X = [0.0, 1.0]
Y = [0.0, 0.5, 2.0]
Z = [0.0, 1.0, 3.0, 4.0]


def tag(i, j, k):
    return 100.0 * i + 10.0 * j + k


def tagged(dims, layout):
    """Values tag(i, j, k) stored in `layout` (z or x fastest)."""
    out = np.zeros(int(np.prod(dims)))
    for i in range(dims[0]):
        for j in range(dims[1]):
            for k in range(dims[2]):
                idx = (i * dims[1] + j) * dims[2] + k if layout == "z" else (k * dims[1] + j) * dims[0] + i
                out[idx] = tag(i, j, k)
    return out


def expected(dims, ncomp):
    """The VTK order: x fastest, components innermost (component c adds c)."""
    return [tag(i, j, k) + c for k in range(dims[2]) for j in range(dims[1]) for i in range(dims[0])
            for c in range(ncomp)]


def arrays(xml):
    out = {}
    for m in re.finditer(r"<DataArray ([^>]*)>(.*?)</DataArray>", xml, re.S):
        attrs = dict(re.findall(r'(\w+)="([^"]*)"', m.group(1)))
        out.setdefault(attrs["Name"], (attrs, m.group(2)))  # the first of a name, as find() does
    return out


def ascii_values(a):
    return [float(t) for t in a[1].split()]


def binary_values(a, header="UInt64"):
    raw = base64.b64decode(a[1].strip())
    hs = 8 if header == "UInt64" else 4
    n = struct.unpack("<Q" if hs == 8 else "<I", raw[:hs])[0]
    body = raw[hs:]
    assert n == len(body)
    fmt = "<f4" if a[0]["type"] == "Float32" else "<f8"
    return list(np.frombuffer(body, dtype=fmt).astype(np.float64))


def well_formed(xml):
    assert xml.startswith('<?xml version="1.0"?>\n')
    names, stack = [], []
    for m in re.finditer(r"<(/?)(\w+)[^>]*?(/?)>", xml):
        if m.group(2) == "xml":
            continue
        if m.group(1):
            assert stack.pop() == m.group(2)
        else:
            names.append(m.group(2))
            if not m.group(3):
                stack.append(m.group(2))
    assert not stack
    return names


def test_structure_and_metadata():
    """vtr/tests.rs:218-274."""
    p = tagged([2, 3, 4], "z")
    c = tagged([1, 2, 3], "z")
    v = np.zeros((24, 3), np.float32)
    s = (V.VtrWriter(X, Y, Z).set_time(1.25e-9).field("Frequency", [2.4e9]).point("p", p).point("E", v)
         .cell("c", c)).to_bytes().decode()
    assert well_formed(s) == ["VTKFile", "RectilinearGrid", "FieldData", "DataArray", "DataArray", "Piece",
                              "PointData", "DataArray", "DataArray", "CellData", "DataArray", "Coordinates",
                              "DataArray", "DataArray", "DataArray"]
    assert '<VTKFile type="RectilinearGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">' in s
    assert '<RectilinearGrid WholeExtent="0 1 0 2 0 3">' in s
    assert '<Piece Extent="0 1 0 2 0 3">' in s
    assert '<PointData Scalars="p" Vectors="E">' in s
    assert '<CellData Scalars="c">' in s
    arrs = arrays(s)
    t = arrs["TimeValue"]
    assert t[0]["NumberOfTuples"] == "1" and t[0]["format"] == "ascii"
    assert ascii_values(t) == [1.25e-9]
    assert ascii_values(arrs["Frequency"]) == [2.4e9]
    assert arrs["E"][0]["type"] == "Float32" and arrs["E"][0]["NumberOfComponents"] == "3"
    assert arrs["E"][0]["format"] == "binary"
    assert arrs["p"][0]["type"] == "Float64"
    for name, co in zip("xyz", (X, Y, Z)):
        assert binary_values(arrs[name]) == co


def test_ascii_round_trip_and_reordering():
    """vtr/tests.rs:276-302: z- and x-fastest inputs give the same file order."""
    dims = [2, 3, 4]
    s = (V.VtrWriter(X, Y, Z, encoding="ascii").point("z", tagged(dims, "z"), "z")
         .point("x", tagged(dims, "x"), "x")).to_bytes().decode()
    arrs = arrays(s)
    assert all(a[0]["format"] == "ascii" for a in arrs.values())
    assert ascii_values(arrs["z"]) == expected(dims, 1)
    assert ascii_values(arrs["x"]) == expected(dims, 1)
    coords = [a for n, a in arrays_all(s) if n in "xyz" and a[0].get("NumberOfComponents") == "1"][-3:]
    assert [ascii_values(c) for c in coords] == [X, Y, Z]


def arrays_all(xml):
    return [(dict(re.findall(r'(\w+)="([^"]*)"', m.group(1)))["Name"],
             (dict(re.findall(r'(\w+)="([^"]*)"', m.group(1))), m.group(2)))
            for m in re.finditer(r"<DataArray ([^>]*)>(.*?)</DataArray>", xml, re.S)]


def test_ascii_exact_floats():
    """vtr/tests.rs:304-324: shortest round-trip text of f64 and f32."""
    x = [0.0, 0.1, 1.0 / 3.0]
    vals = [np.pi, -1e-300, 5e-324]
    vals32 = np.array([0.1, -3.4e38, 1.0 / 3.0], np.float32)
    s = (V.VtrWriter(x, [0.0], [0.0], encoding="ascii").point("a", np.array(vals), "x")
         .point("b", vals32, "x")).to_bytes().decode()
    arrs = arrays(s)
    assert ascii_values(arrs["a"]) == vals
    assert np.array_equal(np.array(arrs["b"][1].split(), dtype=np.float32), vals32)
    assert ascii_values(arrays_all(s)[-3][1]) == x
    assert V.rust_exp(1.0) == "1e0" and V.rust_exp(-0.0025) == "-2.5e-3" and V.rust_exp(0.0) == "0e0"
    assert V.rust_exp(np.float32(0.1), single=True) == "1e-1"


@pytest.mark.parametrize("header", ["UInt64", "UInt32"])
def test_binary_vectors_both_headers(header):
    """vtr/tests.rs:326-358."""
    dims = [2, 3, 4]
    comp = lambda c: (tagged(dims, "z") + c).astype(np.float32)  # noqa: E731
    v = np.stack([comp(0), comp(1), comp(2)], axis=1)
    s = V.VtrWriter(X, Y, Z, header=header).point("E", v).to_bytes().decode()
    assert f'header_type="{header}"' in s
    arrs = arrays(s)
    assert arrs["E"][0]["NumberOfComponents"] == "3"
    assert binary_values(arrs["E"], header) == expected(dims, 3)
    raw = base64.b64decode(arrs["E"][1].strip())
    assert len(raw) == (8 if header == "UInt64" else 4) + 24 * 3 * 4
    assert binary_values(arrs["y"], header) == Y


def test_cell_data_and_planes():
    """vtr/tests.rs:360-392: cell counts, and a plane (one z coordinate)
    counts one flat cell layer."""
    cdims = [1, 2, 3]
    s = V.VtrWriter(X, Y, Z, encoding="ascii").cell("c", tagged(cdims, "z")).to_bytes().decode()
    assert ascii_values(arrays(s)["c"]) == expected(cdims, 1)
    x3, y4 = [0.0, 1.0, 2.0], [0.0, 1.0, 2.0, 3.0]
    pdims, cd = [3, 4, 1], [2, 3, 1]
    cv = np.stack([tagged(cd, "z") + c for c in range(3)], axis=1)
    s = (V.VtrWriter(x3, y4, [0.0], encoding="ascii").point("p", tagged(pdims, "z")).cell("cv", cv)
         .to_bytes().decode())
    assert 'WholeExtent="0 2 0 3 0 0"' in s
    arrs = arrays(s)
    assert ascii_values(arrs["p"]) == expected(pdims, 1)
    assert ascii_values(arrs["cv"]) == expected(cd, 3)


def test_appended_raw():
    """vtr/tests.rs:394-444: offsets contiguous over the appended block."""
    dims = [2, 3, 4]
    for header in ("UInt64", "UInt32"):
        out = (V.VtrWriter(X, Y, Z, encoding="appended", header=header).set_time(3.0)
               .point("p", tagged(dims, "z")).cell("c", tagged([1, 2, 3], "z")).to_bytes())
        tail = b"\n  </AppendedData>\n</VTKFile>\n"
        assert out.endswith(tail)
        head, raw = out.split(b'<AppendedData encoding="raw">\n   _', 1)
        raw = raw[:-len(tail)]
        hs = 8 if header == "UInt64" else 4
        consumed, results = 0, {}
        for m in re.finditer(rb'<DataArray type="(\w+)" Name="(\w+)" NumberOfComponents="\d" format="appended" '
                             rb'offset="(\d+)">', head):
            off = int(m.group(3))
            assert off == consumed
            n = struct.unpack("<Q" if hs == 8 else "<I", raw[off:off + hs])[0]
            results[m.group(2).decode()] = list(np.frombuffer(raw[off + hs:off + hs + n], "<f8"))
            consumed = off + hs + n
        assert consumed == len(raw)
        assert results["p"] == expected(dims, 1)
        assert results["c"] == expected([1, 2, 3], 1)
        assert results["x"] == X and results["z"] == Z


def test_complex_arrays():
    """vtr/tests.rs:446-510: re/im and mag/phase splits."""
    re_ = np.array([3.0, 0.0, -1.0])
    im_ = np.array([4.0, 2.0, 0.0])
    s = (V.VtrWriter([0.0, 1.0, 2.0], [0.0], [0.0], encoding="ascii").point_complex("V", re_, im_)
         .point_complex("W", re_, im_, form="magphase")).to_bytes().decode()
    arrs = arrays(s)
    assert ascii_values(arrs["V_re"]) == list(re_) and ascii_values(arrs["V_im"]) == list(im_)
    assert ascii_values(arrs["W_mag"]) == [5.0, 2.0, 1.0]
    assert np.allclose(ascii_values(arrs["W_phase"]), np.arctan2(im_, re_), atol=1e-15)


def test_validation_errors():
    """vtr/tests.rs:512-560: nothing is written for invalid input."""
    g = lambda: V.VtrWriter(X, Y, Z)  # noqa: E731
    bad = [
        g().point("p", np.zeros(23)),
        g().point("", np.zeros(24)),
        g().point("p", np.zeros(24)).point("p", np.zeros(24)),
        g().cell("c", np.zeros(5)),
        g().point("v", np.zeros((23, 3), np.float32)),
        V.VtrWriter([0.0, 0.0], Y, Z).point("p", np.zeros(24)),
        V.VtrWriter([], Y, Z),
        g().set_time(1.0).field("TimeValue", [1.0]),
        g().field("", [1.0]),
    ]
    for w in bad:
        with pytest.raises(ValueError):
            w.to_bytes()
    with pytest.raises(ValueError):
        V.PvdCollection().push(float("nan"), "a.vtr").to_bytes()


def test_dump_files(tmp_path):
    """tests/dump.rs:444-489: a time series every 10 states and a
    frequency dump, sampled on the oracle."""
    m = analytic_model()
    o = OracleEngine(m, threads=1)
    set_analytic(o, m)
    s = E.Sampler(m, E.DUMP_E, E.NODES, [0, 0, 1], [4, 4, 1], stride=[2, 1, 1])
    states, vals = [], []
    for st in range(31):
        if st:
            o.run(1)
        if st % 10 == 0:
            states.append(st)
            vals.append(o.sample(s))
    V.write_time_dump(s, states, vals, m.dt, str(tmp_path / "td"), "E")
    pvd = (tmp_path / "td" / "E.pvd").read_text()
    assert pvd.count("<DataSet ") == 4
    assert 'file="E_00000030.vtr"' in pvd
    x = (tmp_path / "td" / "E_00000010.vtr").read_text()
    assert '<RectilinearGrid WholeExtent="0 2 0 4 0 0">' in x
    assert 'Name="E"' in x and 'NumberOfComponents="3"' in x and "TimeValue" in x
    assert x.rstrip().endswith("</VTKFile>")
    got = binary_values(arrays(x)["E"])
    want = np.asarray(vals[1], np.float64).reshape(3, 5, 1, 3).transpose(2, 1, 0, 3).astype(np.float32).ravel()
    assert got == list(want.astype(np.float64))
    freqs = [1e9, 2e9]
    V.write_freq_dump(s, freqs, [np.array(vals[0]) * (1 + 1j), np.array(vals[1]) * 1j], str(tmp_path / "fd"), "Ef")
    pvd = (tmp_path / "fd" / "Ef.pvd").read_text()
    assert pvd.count("<DataSet ") == 2 and 'file="Ef_f1.vtr"' in pvd
    f0 = (tmp_path / "fd" / "Ef_f0.vtr").read_text()
    assert 'Name="E_re"' in f0 and 'Name="E_im"' in f0 and 'Name="Frequency"' in f0
    assert 'WholeExtent="0 2 0 4 0 0"' in f0
    assert sorted(os.listdir(tmp_path / "fd")) == ["Ef.pvd", "Ef_f0.vtr", "Ef_f1.vtr"]
