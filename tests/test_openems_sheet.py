"""openEMS's conducting-sheet model for files (ems_b200/openems_sheet.py and
the sheet edges of ems_b200/openems.py) against the reference's own unit
vectors (src/compile/openems_sheet.rs tests `bins`, `capacitance_is_openems`,
`thin_sheets_conduct_sigma_t`) and the branch constants the host installs
(src/engine/openems_sheet.rs:56-80). The fixture runs against openEMS's
output are in test_openems_fixtures.py. CPU only.
"""
from __future__ import annotations

import ctypes as _C
import math
import struct

import numpy as np
import pytest

import ems_b200 as E
from ems_b200 import openems as OE
from ems_b200 import openems_sheet as OS

MU0 = 4e-7 * math.pi
C_u8, C_f64, C_u64 = _C.c_uint8, _C.c_double, _C.c_uint64


def test_bins_of_the_reference_test():
    s, t = 5.8e7, 3.5e-5  # copper, 35 um: bin 9 between 7.3094 and 10.965 GHz
    assert OS.bin_index(s, t, 7.30e9) == 8
    assert OS.bin_index(s, t, 7.32e9) == 9
    assert OS.bin_index(s, t, 10.95e9) == 9
    assert OS.bin_index(s, t, 10.98e9) == 10
    assert OS.bin_index(s, t, 0.0) == 0
    assert OS.bin_index(1e3, 1e-5, 1e12) == 0
    assert OS.bin_index(s, 1.0, 1e12) == 29
    f = 80.0 / (math.pi * MU0 * 1e6 * 4e-10)  # t/delta = sqrt(80): the edge of bin 0
    assert OS.bin_index(1e6, 2e-5, f * 0.9999) == 0
    assert OS.bin_index(1e6, 2e-5, f * 1.0001) == 1
    # Bin edges one f32 step of f apart, measured on openEMS.
    for s_, t_, f_lo, f_hi, k in [
            (4613344.0, 1.526974870103004e-06, 1883868758016.0, 1883868889088.0, 1),
            (22566374.0, 2.323430271644611e-05, 1663447680.0, 1663447808.0, 1),
            (27018.404296875, 7.05397324054502e-05, 3863073521664.0, 3863073783808.0, 9),
            (10959826.0, 4.6812994696665555e-05, 72978948096.0, 72978956288.0, 12),
            (10243358.0, 3.557360469130799e-05, 3465501474816.0, 3465501736960.0, 20)]:
        assert OS.bin_index(s_, t_, f_lo) == k - 1
        assert OS.bin_index(s_, t_, f_hi) == k


def test_capacitance_is_openems():
    """openEMS's vi = f32(dt/f32(C)) of a 1 m-cell sheet edge (bin 0),
    from its operator dumps."""
    s, t = 9.536741259755848e-07, 6.090221230296086e-05
    for dt, vi in [(1.8108346533866837e-09, 0x3a763a62), (3.5948730289534073e-10, 0x3b9b0a27),
                   (1.807569004847039e-09, 0x3a76ac43)]:
        _, c_dt2, _ = OS.edge_circuit(s, t, 1.0, OS.TABLE[OS.bin_index(s, t, 1e6)])
        c = c_dt2 * dt * dt
        got = np.float32(dt / float(np.float32(c)))
        assert struct.unpack("<I", struct.pack("<f", got))[0] == vi


def test_thin_sheets_conduct_sigma_t():
    row = OS.TABLE[0]
    assert abs(row[0] + 1.0 / row[3] + 1.0 / row[5] - 1.0) < 2e-3


SHEET_XML = """<?xml version="1.0" encoding="UTF-8"?>
<openEMS>
  <FDTD NumberOfTimesteps="50" endCriteria="1e-30">
    <Excitation Type="0" f0="4e9" fc="4e9"/>
    <BoundaryCond xmin="PEC" xmax="PEC" ymin="MUR" ymax="PML_3" zmin="PEC" zmax="PEC"/>
  </FDTD>
  <ContinuousStructure CoordSystem="0">
    <Properties>
      <Excitation Name="exc" Type="0" Excite="0,0,1"><Primitives><Box Priority="0"><P1 X="3" Y="8" Z="4"/><P2 X="3" Y="8" Z="6"/></Box></Primitives></Excitation>
      <ConductingSheet Name="s" Conductivity="5.8e7" Thickness="3.5e-5"><Primitives><Box Priority="0"><P1 X="6" Y="0" Z="2"/><P2 X="6" Y="14" Z="8"/></Box></Primitives></ConductingSheet>
      <ProbeBox Name="u" Type="0"><Primitives><Box Priority="0"><P1 X="9" Y="6" Z="3"/><P2 X="9" Y="6" Z="7"/></Box></Primitives></ProbeBox>
    </Properties>
    <RectilinearGrid DeltaUnit="1e-3" CoordSystem="0">
      <XLines>0,1,2,3,4,5,6,7,8,9,10,11,12</XLines>
      <YLines>0,1,2,3,4,5,6,7,8,9,10,11,12,13,14,15,16</YLines>
      <ZLines>0,1,2,3,4,5,6,7,8,9,10</ZLines>
    </RectilinearGrid>
  </ContinuousStructure>
</openEMS>
"""


def test_sheet_edges_widths_pec_rows_and_branch_constants():
    """The sheet on x = 6: its y and z edges between the sheet's borders
    are sheet edges, the edges whose node lies on the lines that the Mur
    face (y = 0, 1) or the PML_3 face (the last four y lines) claims, and
    those in the first cell of their axis, are PEC; an edge on the sheet's
    border row carries half the width (one neighbouring cell outside the
    sheet). Each sheet edge gets the circuit's C and G (its coefficients)
    and two sheet-branch poles whose constants are the reference's
    ka = f32((L/dt - R/2)/(L/dt + R/2)), kb = f32(cb/(L/dt + R/2))."""
    s = OE.loads(SHEET_XML)
    m, dt = s.model, s.dt
    n = s.nodes
    edges = {(a, (i, j, k)) for a, i, j, k in s.sheet_edges}
    assert all(i == 6 for _, (i, _, _) in edges)
    ys = sorted({j for a, (_, j, _) in edges if a == 2})
    assert ys[0] == 2 and ys[-1] == n[1] - 1 - 4  # y = 0, 1 (Mur) and the last four lines (PML_3) left out
    row = OS.TABLE[OS.bin_index(5.8e7, 3.5e-5, 8e9)]
    checked = 0
    for a, node, branches in s.sheet_branches:
        # z edges along y = 8: full width across y; y edges: full width
        # across z, half on the sheet's border rows z = 2 and z = 8 (one
        # neighbouring cell off the sheet).
        if a == 2 and node[1] == 8:
            t, half = 1, False
        elif a == 1 and node[1] == 7:
            t, half = 2, node[2] in (2, 8)
        else:
            continue
        width = s.model_dual(t, node[t]) * (0.5 if half else 1.0)
        br, c_dt2, g = OS.edge_circuit(5.8e7, 3.5e-5, s.model_delta(a, node[a]) / width, row)
        assert br == branches, (a, node)
        cap, cond = float(np.float32(c_dt2 * dt * dt)), float(np.float32(g))
        assert m.coeff(3 + a)[node] == np.float32(dt / (cap + 0.5 * cond * dt))
        checked += 1
    assert checked == 6 + 7
    # The branch constants in the engine's pole table.
    d = E.EngineDesc.from_address(m.desc)
    ops = (E.OpEntry * d.n_ops).from_address(d.ops)
    poles = next(E.PolesTable.from_address(o.table) for o in ops if o.kind == E.OP_POLES)
    pe = poles.electric
    ne, npl = int(pe.n_edges), int(pe.n_poles)
    assert ne == len(s.sheet_branches) and npl == 2 * ne
    kind = np.ctypeslib.as_array((C_u8 * npl).from_address(pe.kind))
    a_ = np.ctypeslib.as_array((C_f64 * npl).from_address(pe.a))
    ic = np.ctypeslib.as_array((C_f64 * npl).from_address(pe.inv_c))
    iz = np.ctypeslib.as_array((C_f64 * npl).from_address(pe.inv_z))
    node = np.ctypeslib.as_array((C_u64 * ne).from_address(pe.node))
    axis = np.ctypeslib.as_array((C_u8 * ne).from_address(pe.axis))
    assert np.all(kind == 2) and np.all(ic == 0.0)  # openEMS f32 poles, no restoring term
    by_edge = {(int(axis[e]), int(node[e])): e for e in range(ne)}
    for a, nd, branches in s.sheet_branches:
        flat = (nd[0] * n[1] + nd[1]) * n[2] + nd[2]
        e = by_edge[(a, flat)]
        cbe = float(m.coeff(3 + a)[nd])
        for q, (ind, res) in enumerate(branches):
            den = ind / dt + 0.5 * res
            assert a_[2 * e + q] == float(np.float32((ind / dt - 0.5 * res) / den))
            assert iz[2 * e + q] == float(np.float32(cbe / den))


def test_refusals():
    bad = SHEET_XML.replace('<P1 X="6" Y="0" Z="2"/><P2 X="6" Y="14" Z="8"/>',
                            '<P1 X="6.5" Y="0" Z="2"/><P2 X="6.5" Y="14" Z="8"/>')
    with pytest.raises(NotImplementedError):
        OE.loads(bad)
    thick = SHEET_XML.replace('<P2 X="6" Y="14" Z="8"/>', '<P2 X="7" Y="14" Z="8"/>')
    with pytest.raises(NotImplementedError):
        OE.loads(thick)
