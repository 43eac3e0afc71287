"""openEMS XML models on the CUDA engine against the oracle.

Models written for this test in openEMS's XML (graded meshes, PEC, PMC and
Mur faces, anisotropic lossy materials with magnetic conductivity, metal
under a higher-priority material, a parallel R/C lumped element, Lorentz, Drude, magnetic and Debye
poles, soft and hard E and H excitations with every signal type and a
delay, voltage, current, E and H field probes with FD samples, a time
window and a probe oversampling, an energy end criterion) are set up by
ems_b200/openems.py and run on the CUDA engine (every schedule that can
run them) and on the oracle: every probe series, every written probe file
and the final fields agree bit for bit. The oracle itself is checked
against openEMS's own output for the same features in
test_openems_fixtures.py. Also the command-line entry point.
"""
import math
import os

import numpy as np
import pytest

import ems_b200 as E
from ems_b200 import openems as OE
from helpers import assert_fields_equal
from oracle import OracleEngine

pytestmark = pytest.mark.gpu


def _lines(v):
    return ",".join(f"{x:g}" for x in v)


X = [0, 1, 2, 3, 4, 5, 5.5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16]
Y = [0, 1, 2, 3, 4, 4.6, 5.2, 6, 7, 8, 9, 10, 11, 12, 13]
Z = [0, 1.2, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12]

BOX = f"""<?xml version="1.0" encoding="UTF-8"?>
<openEMS>
  <FDTD NumberOfTimesteps="420" endCriteria="1e-30" OverSampling="3">
    <Excitation Type="0" f0="4e9" fc="3e9"/>
    <BoundaryCond xmin="PEC" xmax="MUR" ymin="PMC" ymax="PEC" zmin="MUR" zmax="PEC" MUR_PhaseVelocity="2.6e8"/>
  </FDTD>
  <ContinuousStructure CoordSystem="0">
    <Properties>
      <Material Name="aniso" Isotropy="0"><Property Epsilon="2,3.5,2.5" Mue="1,1.4,1.2" Kappa="0.01,0.005,0.02" Sigma="80,0,40"/>
        <Primitives><Box Priority="1"><P1 X="9" Y="2" Z="2"/><P2 X="14" Y="9" Z="7"/></Box></Primitives></Material>
      <Metal Name="block"><Primitives><Box Priority="2"><P1 X="10" Y="4" Z="3"/><P2 X="12" Y="6" Z="5"/></Box></Primitives></Metal>
      <Material Name="over"><Property Epsilon="4" Kappa="0.01"/>
        <Primitives><Box Priority="3"><P1 X="10" Y="4" Z="5"/><P2 X="12" Y="6" Z="6"/></Box></Primitives></Material>
      <LumpedElement Name="rc" Direction="2" R="75" C="2e-13" Caps="1"><Primitives><Box Priority="5"><P1 X="2" Y="9" Z="4"/><P2 X="3" Y="10" Z="7"/></Box></Primitives></LumpedElement>
      <Excitation Name="soft" Type="0" Excite="0.3,0,1"><Primitives><Box Priority="0"><P1 X="4" Y="7" Z="5"/><P2 X="5" Y="7" Z="7"/></Box></Primitives></Excitation>
      <Excitation Name="hard" Type="1" Excite="0,0.5,0"><Primitives><Box Priority="0"><P1 X="15" Y="10" Z="9"/><P2 X="15" Y="11" Z="9"/></Box></Primitives></Excitation>
      <ProbeBox Name="ut" Type="0"><FD_Samples>2e9,4e9,6e9</FD_Samples><Primitives><Box Priority="0"><P1 X="7" Y="7" Z="4"/><P2 X="7" Y="7" Z="8.4"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="ur" Type="0" Weight="-2"><Primitives><Box Priority="0"><P1 X="13" Y="8" Z="3"/><P2 X="9.6" Y="8" Z="3"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="it" Type="1" NormDir="2"><FD_Samples>3e9</FD_Samples><Primitives><Box Priority="0"><P1 X="3" Y="5.2" Z="6.3"/><P2 X="6" Y="9" Z="6.3"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="ix" Type="1"><Primitives><Box Priority="0"><P1 X="8" Y="3" Z="2"/><P2 X="8" Y="10" Z="9"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="ef" Type="2" StartTime="1e-10" StopTime="5e-10"><Primitives><Box Priority="0"><P1 X="8" Y="7" Z="6"/><P2 X="8" Y="7" Z="6"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="hf" Type="3" OverSampling="6"><FD_Samples>4e9</FD_Samples><Primitives><Box Priority="0"><P1 X="5.5" Y="6.5" Z="6"/><P2 X="5.5" Y="6.5" Z="6"/></Box></Primitives></ProbeBox>
    </Properties>
    <RectilinearGrid DeltaUnit="0.001" CoordSystem="0">
      <XLines>{_lines(X)}</XLines>
      <YLines>{_lines(Y)}</YLines>
      <ZLines>{_lines(Z)}</ZLines>
    </RectilinearGrid>
  </ContinuousStructure>
</openEMS>
"""

SINE = f"""<?xml version="1.0" encoding="UTF-8"?>
<openEMS>
  <FDTD NumberOfTimesteps="300" endCriteria="-1" TimeStepFactor="0.9">
    <Excitation Type="1" f0="3e9"/>
    <BoundaryCond xmin="PMC" xmax="PEC" ymin="PEC" ymax="PMC" zmin="PEC" zmax="MUR"/>
  </FDTD>
  <ContinuousStructure CoordSystem="0">
    <BackgroundMaterial Epsilon="1.5" Mue="1.1"/>
    <Properties>
      <Excitation Name="h" Type="2" Excite="0,0,1" Delay="1.3e-10"><Primitives><Box Priority="0"><P1 X="6.5" Y="5.5" Z="6"/><P2 X="7.5" Y="6.5" Z="6"/></Box></Primitives></Excitation>
      <Excitation Name="off" Type="0" Excite="1,0,0" Enabled="0"><Primitives><Box Priority="0"><P1 X="2" Y="2" Z="2"/><P2 X="3" Y="2" Z="2"/></Box></Primitives></Excitation>
      <ProbeBox Name="hz" Type="3"><FD_Samples>3e9</FD_Samples><Primitives><Box Priority="0"><P1 X="8.5" Y="6.5" Z="6.5"/><P2 X="8.5" Y="6.5" Z="6.5"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="ue" Type="0"><Primitives><Box Priority="0"><P1 X="9" Y="4" Z="6"/><P2 X="9" Y="8" Z="6"/></Box></Primitives></ProbeBox>
    </Properties>
    <RectilinearGrid DeltaUnit="0.001" CoordSystem="0">
      <XLines>{_lines(X)}</XLines>
      <YLines>{_lines(Y)}</YLines>
      <ZLines>{_lines(Z)}</ZLines>
    </RectilinearGrid>
  </ContinuousStructure>
</openEMS>
"""

PULSES = f"""<?xml version="1.0" encoding="UTF-8"?>
<openEMS>
  <FDTD NumberOfTimesteps="90" endCriteria="1e-30" TimeStepMethod="1">
    <Excitation Type="10" f0="5e9" Function="exp(-((t-6e-11)/2e-11)^2)*sin(2*pi*5e9*t)"/>
    <BoundaryCond xmin="PEC" xmax="PEC" ymin="PEC" ymax="PEC" zmin="PEC" zmax="PEC"/>
  </FDTD>
  <ContinuousStructure CoordSystem="0">
    <Properties>
      <Excitation Name="hh" Type="3" Excite="0,1,0"><Primitives><Box Priority="0"><P1 X="5.5" Y="6" Z="5.5"/><P2 X="5.5" Y="6" Z="5.5"/></Box></Primitives></Excitation>
      <Excitation Name="se" Type="0" Excite="0,0,-1"><Primitives><Box Priority="0"><P1 X="9" Y="8" Z="3"/><P2 X="9" Y="8" Z="6"/></Box></Primitives></Excitation>
      <ProbeBox Name="e" Type="2"><Primitives><Box Priority="0"><P1 X="7" Y="7" Z="5"/><P2 X="8" Y="8" Z="6"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="i" Type="1" NormDir="1"><Primitives><Box Priority="0"><P1 X="4" Y="6.4" Z="4"/><P2 X="7" Y="6.4" Z="7"/></Box></Primitives></ProbeBox>
    </Properties>
    <RectilinearGrid DeltaUnit="0.001" CoordSystem="0">
      <XLines>{_lines(X)}</XLines>
      <YLines>{_lines(Y)}</YLines>
      <ZLines>{_lines(Z)}</ZLines>
    </RectilinearGrid>
  </ContinuousStructure>
</openEMS>
"""


DISP = f"""<?xml version="1.0" encoding="UTF-8"?>
<openEMS>
  <FDTD NumberOfTimesteps="360" endCriteria="1e-4" f_max="10e9">
    <Excitation Type="0" f0="5e9" fc="4e9"/>
    <BoundaryCond xmin="PEC" xmax="PEC" ymin="PMC" ymax="PMC" zmin="PEC" zmax="PEC"/>
  </FDTD>
  <ContinuousStructure CoordSystem="0">
    <Properties>
      <LorentzMaterial Name="lor" Order="2">
        <Property Epsilon="2" Mue="1.2" EpsilonPlasmaFrequency_1="5e9" EpsilonLorPoleFrequency_1="7e9" EpsilonRelaxTime_1="1e-9"
                  EpsilonPlasmaFrequency_2="3e9" EpsilonRelaxTime_2="2e-10" MuePlasmaFrequency_2="2e9" MueRelaxTime_2="5e-10"/>
        <Primitives><Box Priority="1"><P1 X="8" Y="2" Z="2"/><P2 X="12.5" Y="9" Z="8"/></Box></Primitives></LorentzMaterial>
      <DebyeMaterial Name="deb" Order="1"><Property Epsilon="1.5" EpsilonDelta_1="2" EpsilonRelaxTime_1="3e-11"/>
        <Primitives><Box Priority="2"><P1 X="11" Y="4" Z="3"/><P2 X="14" Y="7" Z="6"/></Box></Primitives></DebyeMaterial>
      <Excitation Name="soft" Type="0" Excite="0,0,1"><Primitives><Box Priority="0"><P1 X="4" Y="6" Z="4"/><P2 X="4" Y="6" Z="7"/></Box></Primitives></Excitation>
      <ProbeBox Name="ut" Type="0"><Primitives><Box Priority="0"><P1 X="10" Y="6" Z="3"/><P2 X="10" Y="6" Z="7"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="it" Type="1" NormDir="0"><Primitives><Box Priority="0"><P1 X="13" Y="3" Z="2"/><P2 X="13" Y="9" Z="8"/></Box></Primitives></ProbeBox>
    </Properties>
    <RectilinearGrid DeltaUnit="0.001" CoordSystem="0">
      <XLines>{_lines(X)}</XLines>
      <YLines>{_lines(Y)}</YLines>
      <ZLines>{_lines(Z)}</ZLines>
    </RectilinearGrid>
  </ContinuousStructure>
</openEMS>
"""


PMLM = f"""<?xml version="1.0" encoding="UTF-8"?>
<openEMS>
  <FDTD NumberOfTimesteps="600" endCriteria="0.05">
    <Excitation Type="0" f0="8e9" fc="6e9"/>
    <BoundaryCond xmin="PEC" xmax="PML_5" ymin="PML_4" ymax="PMC" zmin="PEC" zmax="PML_3"/>
  </FDTD>
  <ContinuousStructure CoordSystem="0">
    <Properties>
      <Material Name="block"><Property Epsilon="2.2" Mue="1.3" Kappa="0.02" Sigma="30"/>
        <Primitives><Box Priority="1"><P1 X="9" Y="0" Z="5"/><P2 X="16" Y="6" Z="12"/></Box></Primitives></Material>
      <Excitation Name="exc" Type="0" Excite="0.3,0.5,1"><Primitives><Box Priority="0"><P1 X="5" Y="7" Z="4"/><P2 X="6" Y="8" Z="6"/></Box></Primitives></Excitation>
      <ProbeBox Name="ut" Type="0"><Primitives><Box Priority="0"><P1 X="8" Y="6" Z="0"/><P2 X="8" Y="6" Z="12"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="ein" Type="2"><Primitives><Box Priority="0"><P1 X="14" Y="2" Z="10"/><P2 X="14" Y="2" Z="10"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="hin" Type="3"><Primitives><Box Priority="0"><P1 X="15" Y="1" Z="11"/><P2 X="15" Y="1" Z="11"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="it" Type="1" NormDir="0"><Primitives><Box Priority="0"><P1 X="12" Y="2" Z="2"/><P2 X="12" Y="10" Z="10"/></Box></Primitives></ProbeBox>
    </Properties>
    <RectilinearGrid DeltaUnit="0.001" CoordSystem="0">
      <XLines>{_lines(X)}</XLines>
      <YLines>{_lines(Y)}</YLines>
      <ZLines>{_lines(Z)}</ZLines>
    </RectilinearGrid>
  </ContinuousStructure>
</openEMS>
"""


# openEMS's conducting-sheet model: a copper sheet on the plane x = 8 (a
# lumped resistor partly on it, a hard E source across it), a resistive
# sheet on z = 5 under a Lorentz block and a metal strip of lower priority,
# PMC faces (the H edges next to sheet edges kept).
SHEET = f"""<?xml version="1.0" encoding="UTF-8"?>
<openEMS>
  <FDTD NumberOfTimesteps="400" endCriteria="1e-30">
    <Excitation Type="0" f0="5e9" fc="4e9"/>
    <BoundaryCond xmin="PEC" xmax="PEC" ymin="PMC" ymax="PMC" zmin="PEC" zmax="PEC"/>
  </FDTD>
  <ContinuousStructure CoordSystem="0">
    <Properties>
      <LorentzMaterial Name="lor"><Property Epsilon="2.0" EpsilonPlasmaFrequency="5e9" EpsilonLorPoleFrequency="8e9" EpsilonRelaxTime="1e-9"/>
        <Primitives><Box Priority="2"><P1 X="10" Y="2" Z="5"/><P2 X="14" Y="9" Z="8"/></Box></Primitives></LorentzMaterial>
      <Metal Name="strip"><Primitives><Box Priority="1"><P1 X="11" Y="3" Z="5"/><P2 X="13" Y="5" Z="5"/></Box></Primitives></Metal>
      <ConductingSheet Name="cu" Conductivity="5.8e7" Thickness="3.5e-5">
        <Primitives><Box Priority="3"><P1 X="8" Y="2" Z="2"/><P2 X="8" Y="10" Z="10"/></Box></Primitives></ConductingSheet>
      <ConductingSheet Name="res" Conductivity="1e4" Thickness="1e-5">
        <Primitives><Box Priority="3"><P1 X="9" Y="1" Z="5"/><P2 X="15" Y="11" Z="5"/></Box></Primitives></ConductingSheet>
      <LumpedElement Name="r1" Direction="2" Caps="1" R="75"><Primitives><Box Priority="0"><P1 X="8" Y="4.6" Z="4"/><P2 X="9" Y="4.6" Z="7"/></Box></Primitives></LumpedElement>
      <Excitation Name="exc" Type="1" Excite="0,1,0"><Primitives><Box Priority="0"><P1 X="7" Y="6" Z="6"/><P2 X="9" Y="7" Z="6"/></Box></Primitives></Excitation>
      <Excitation Name="soft" Type="0" Excite="0,0,1"><Primitives><Box Priority="0"><P1 X="4" Y="5.2" Z="3"/><P2 X="4" Y="5.2" Z="6"/></Box></Primitives></Excitation>
      <ProbeBox Name="ut" Type="0"><Primitives><Box Priority="0"><P1 X="12" Y="6" Z="0"/><P2 X="12" Y="6" Z="12"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="e8" Type="2"><Primitives><Box Priority="0"><P1 X="8" Y="7" Z="6"/><P2 X="8" Y="7" Z="6"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="h" Type="3"><Primitives><Box Priority="0"><P1 X="13" Y="4" Z="9"/><P2 X="13" Y="4" Z="9"/></Box></Primitives></ProbeBox>
    </Properties>
    <RectilinearGrid DeltaUnit="0.001" CoordSystem="0">
      <XLines>{_lines(X)}</XLines>
      <YLines>{_lines(Y)}</YLines>
      <ZLines>{_lines(Z)}</ZLines>
    </RectilinearGrid>
  </ContinuousStructure>
</openEMS>
"""


# Lumped elements with an inductor or in series (openEMS's order; the
# explicit f32 inductor of a parallel L and of a parallel R||L whose edge
# capacitance openEMS limits; series RLC and series R branches), soft
# sources on two of them, PMC walls across one.
LUMPED = f"""<?xml version="1.0" encoding="UTF-8"?>
<openEMS>
  <FDTD NumberOfTimesteps="400" endCriteria="1e-30">
    <Excitation Type="0" f0="3e9" fc="2e9"/>
    <BoundaryCond xmin="PEC" xmax="PEC" ymin="PEC" ymax="PEC" zmin="PMC" zmax="PMC"/>
  </FDTD>
  <ContinuousStructure CoordSystem="0">
    <Properties>
      <Material Name="sub"><Property Epsilon="3.0" Kappa="0.01"/>
        <Primitives><Box Priority="1"><P1 X="0" Y="0" Z="0"/><P2 X="16" Y="13" Z="3"/></Box></Primitives></Material>
      <LumpedElement Name="pl" Direction="2" Caps="1" L="3e-9"><Primitives><Box Priority="0"><P1 X="4" Y="4" Z="3"/><P2 X="5" Y="4" Z="6"/></Box></Primitives></LumpedElement>
      <LumpedElement Name="prl" Direction="2" Caps="1" R="60" L="2e-9"><Primitives><Box Priority="0"><P1 X="10" Y="4" Z="4"/><P2 X="10" Y="4" Z="7"/></Box></Primitives></LumpedElement>
      <LumpedElement Name="srlc" Direction="1" Caps="0" LEtype="1" R="25" L="2e-9" C="1e-12"><Primitives><Box Priority="0"><P1 X="7" Y="7" Z="5"/><P2 X="7" Y="9" Z="5"/></Box></Primitives></LumpedElement>
      <LumpedElement Name="sr" Direction="2" Caps="1" LEtype="1" R="80"><Primitives><Box Priority="0"><P1 X="13" Y="9" Z="0"/><P2 X="13" Y="9" Z="2"/></Box></Primitives></LumpedElement>
      <Excitation Name="e1" Type="0" Excite="0,0,1"><Primitives><Box Priority="0"><P1 X="10" Y="4" Z="4"/><P2 X="10" Y="4" Z="7"/></Box></Primitives></Excitation>
      <Excitation Name="e2" Type="0" Excite="0,1,0"><Primitives><Box Priority="0"><P1 X="7" Y="7" Z="5"/><P2 X="7" Y="9" Z="5"/></Box></Primitives></Excitation>
      <ProbeBox Name="u_pl" Type="0"><Primitives><Box Priority="0"><P1 X="4" Y="4" Z="3"/><P2 X="4" Y="4" Z="6"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="u_s" Type="0"><Primitives><Box Priority="0"><P1 X="7" Y="7" Z="5"/><P2 X="7" Y="9" Z="5"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="u_sr" Type="0"><Primitives><Box Priority="0"><P1 X="13" Y="9" Z="0"/><P2 X="13" Y="9" Z="2"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="h" Type="3"><Primitives><Box Priority="0"><P1 X="8" Y="6" Z="8"/><P2 X="8" Y="6" Z="8"/></Box></Primitives></ProbeBox>
    </Properties>
    <RectilinearGrid DeltaUnit="0.001" CoordSystem="0">
      <XLines>{_lines(X)}</XLines>
      <YLines>{_lines(Y)}</YLines>
      <ZLines>{_lines(Z)}</ZLines>
    </RectilinearGrid>
  </ContinuousStructure>
</openEMS>
"""


# An absorbing sheet (AbsorbingBC) across the lumped model, absorbing
# waves along -x at the local medium velocity.
ABC = LUMPED.replace("</Properties>", """  <AbsorbingBC Name="abc" NormalSignPositive="1" PhaseVelocity="0">
        <Primitives><Box Priority="0"><P1 X="12" Y="0" Z="0"/><P2 X="12" Y="13" Z="12"/></Box></Primitives></AbsorbingBC>
    </Properties>""")


# Waveguide mode probes (voltage and current, a sine and a step mode
# function) on the lumped model's grid.
WG = LUMPED.replace("</Properties>", """  <ProbeBox Name="wv" Type="10" Weight="2" NormDir="2"><Attributes ModeFunctionX="0" ModeFunctionY="sin(3.14159265*x/16)" ModeFunctionZ="0"/>
        <Primitives><Box Priority="0"><P1 X="0" Y="0" Z="7"/><P2 X="16" Y="13" Z="7"/></Box></Primitives></ProbeBox>
      <ProbeBox Name="wi" Type="11" Weight="-1" NormDir="2"><Attributes ModeFunctionX="(y&gt;4)*(y&lt;9)" ModeFunctionY="0" ModeFunctionZ="0"/>
        <Primitives><Box Priority="0"><P1 X="2" Y="1" Z="8"/><P2 X="14" Y="12" Z="8"/></Box></Primitives></ProbeBox>
    </Properties>""")


def _both(text, schedule=0):
    """Both engines on the model, in openEMS's curl order except on the
    fused and two-kernel schedules, which have only the default one."""
    s = OE.loads(text)
    g = E.Engine(s.model)
    g.set_schedule(schedule)
    o = OracleEngine(s.model, threads=2)
    order = 0 if schedule in (2, 3) else 1
    return s, g, s.run(g, order), o, s.run(o, order)


# Schedules 2 (fused) and 5 (sweep) do not run magnetic sources, 2 not
# magnetic poles; openEMS PML layers run on schedules 1 and 4 only.
@pytest.mark.parametrize("name,text,schedule", [
    ("box", BOX, 0), ("box", BOX, 1), ("box", BOX, 2), ("box", BOX, 3), ("box", BOX, 5),
    ("sine", SINE, 0), ("sine", SINE, 1), ("sine", SINE, 3), ("pulses", PULSES, 0), ("pulses", PULSES, 1),
    ("disp", DISP, 0), ("disp", DISP, 1), ("disp", DISP, 3), ("disp", DISP, 5),
    ("pml", PMLM, 0), ("pml", PMLM, 1), ("pml", PMLM, 4),
    ("sheet", SHEET, 0), ("sheet", SHEET, 1), ("sheet", SHEET, 3),
    ("lumped", LUMPED, 0), ("lumped", LUMPED, 1), ("lumped", LUMPED, 3), ("abc", ABC, 0), ("abc", ABC, 1),
    ("wg", WG, 0), ("wg", WG, 4)])
def test_openems_models_bit_exact(name, text, schedule):
    s, g, rg, o, ro = _both(text, schedule)
    assert s.steps > 0 and s.probes
    if name == "pml":
        assert s.stopped  # the end criterion, with the layers' energy correction
    for p in s.probes:
        a, b = rg.series[p.name], ro.series[p.name]
        assert a.shape == b.shape and a.size
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), (name, p.name)
    assert rg.files().keys() == ro.files().keys()
    for k, text_g in rg.files().items():
        assert text_g.splitlines()[1:] == ro.files()[k].splitlines()[1:], (name, k)
    assert_fields_equal(g, o, f"openEMS model {name}")
    assert any(np.any(v != 0) for v in rg.series.values())


@pytest.mark.parametrize("schedule", [1, 2, 3, 4, 5])
def test_openems_pole_arithmetic(schedule):
    """openEMS's f32 pole kinds on every schedule: Lorentz and Drude poles
    (OpenEmsPole) alone, with a trapezoidal Debye pole on the same edges
    (applied first), edges of Debye poles alone (openEMS's Debye update),
    magnetic poles (not on the fused schedule, which has none), beside CPML
    layers: fields bit for bit with the oracle, energies (which leave these
    poles out) within 1e-12."""
    rng = np.random.default_rng(5)
    lines = [np.cumsum(np.concatenate([[0.0], 1e-3 * (1.0 + 0.3 * rng.random(c))])) for c in (16, 13, 21)]
    m = E.Model(*lines)
    m.fill(m.cells().box([3, 3, 3], [12, 10, 17]), m.material(eps_r=2.0, mu_r=1.3, kappa=0.01))
    m.build()
    m.add_cpml([3, 0, 3, 3, 0, 4], kappa_max=1.5, alpha_max=0.02)
    d = E.Dispersive()
    lor = m.cells().box([4, 4, 4], [11, 9, 12])
    d.fill_cells(m, lor, [E.Pole.lorentz(3e10, 2e10, 1e9), E.Pole.drude(2e10, 4e9)])
    d.fill_cells(m, m.cells().box([8, 2, 9], [14, 8, 16]), [E.Pole.debye(1.5, 2e-11), E.Pole.debye(0.7, 5e-11)])
    if schedule != 2:
        d.fill_cells(m, m.cells().box([2, 5, 5], [9, 11, 10]), [E.Pole.drude(1e10, 3e9)], field=1)
    m.add_dispersive(d, E.OPENEMS_POLES)
    f0, fc = 10e9, 8e9
    amp = [math.exp(-((k * m.dt - 1.2e-10) * fc) ** 2) * math.sin(2 * math.pi * f0 * k * m.dt) for k in range(200)]
    m.add_source_table(E.SOFT_E, [(E.Z, (6, 6, 8), 1.0), (E.Y, (10, 5, 12), 0.6)], np.array(amp))
    g = E.Engine(m)
    g.set_schedule(schedule)
    o = OracleEngine(m, threads=2)
    eg, eo = [], []
    for s in range(0, 200, 10):
        eg.append(g.step_with_energy())
        eo.append(o.step_with_energy())
        g.run(9)
        o.run(9)
    assert g.schedule == schedule
    np.testing.assert_allclose(eg, eo, rtol=1e-12, atol=0)
    assert_fields_equal(g, o, f"openEMS pole kinds, schedule {schedule}")


@pytest.mark.parametrize("schedule", [1, 4, 5])
def test_openems_curl_order_with_every_operator(schedule):
    """openEMS's summation order on a model with every operator (CPML,
    electric poles, lumped port, sources, probes): bit for bit with the
    oracle; and it differs from the default order."""
    from helpers import mixed_model

    m, ops = mixed_model(magnetic=False, h_source=False, steps=200)
    g = E.Engine(m)
    g.set_schedule(schedule)
    g.set_curl_order(1)
    with pytest.raises(E.EngineError):
        g.set_schedule(3)
    o = OracleEngine(m, threads=3)
    o.set_curl_order(1)
    g.run(200)
    o.run(200)
    assert_fields_equal(g, o, f"openEMS order, schedule {schedule}")
    for k in (ops["pv"], ops["pe"]):
        assert np.array_equal(g.samples(k).view(np.uint64), o.samples(k).view(np.uint64))
    d = E.Engine(m)
    d.set_schedule(schedule)
    d.run(200)
    assert not np.array_equal(d.field(0, E.Z), g.field(0, E.Z))


def test_openems_command_line(tmp_path):
    path = tmp_path / "model.xml"
    path.write_text(BOX)
    assert OE.main([str(path), str(tmp_path / "out")]) == 0
    s = OE.loads(BOX)
    ro = s.run(OracleEngine(s.model, threads=2))
    want = {**ro.files(), **ro.signal_files()}
    assert sorted(os.listdir(tmp_path / "out")) == sorted(want)
    for k, text in want.items():
        assert (tmp_path / "out" / k).read_text().splitlines()[1:] == text.splitlines()[1:], k
