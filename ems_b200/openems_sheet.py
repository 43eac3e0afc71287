"""openEMS's conducting-sheet model for openEMS files (the reference's
src/compile/openems_sheet.rs and src/engine/openems_sheet.rs).

openEMS v0.37 does not model a ``ConductingSheet`` as a thin slab (the
engine's own sheet, ``ems_model_add_sheet``) but with a fitted edge
circuit, which the reference reproduces for files as measured on openEMS:
each sheet edge is a capacitor ``C`` with a conductance ``G`` in parallel
with two series R-L branches, ``C·du/dt + G·u + Σ i_b = I``,
``L_b·di_b/dt + R_b·i_b = u``, the branches integrated in openEMS's single
precision like its Drude poles. Per square of sheet ``G = g·σt``,
``R_b = r_b/(σt)``, ``L_b = l_b·μ0·t`` and ``C/dt² = 1/(c·μ0·t)``, with
``(g, c, l_1, r_1, l_2, r_2)`` from ``TABLE`` by the bin of the normalised
thickness ``ν = (t/δ)²/80`` at the excitation's highest frequency; an edge
of length ``l`` with sheet width ``w`` has ``w/l`` squares. All the f32
roundings are openEMS's, as the reference measured them.

On the engine the edge's ``C`` and ``G`` replace its medium
(``ems_model_set_edge_circuit``) and each branch is an openEMS f32 pole
step with no restoring term (``Pole.sheet_branch``: ``x ← ka·x + kb·uⁿ``,
``u ← u − x``).
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["TABLE", "OPENEMS_MU0", "sheet_frequency", "bin_index", "edge_circuit"]

OPENEMS_MU0 = 1.256637062e-6  # openEMS's vacuum permeability (src/constants.rs)

# (g, c, l_1, r_1, l_2, r_2) per bin k of ν = (t/δ)²/80: openEMS v0.37's
# fitted sheet model as the reference measured it on openEMS
# (src/compile/openems_sheet.rs:137-170). Data, kept as measured: these are
# openEMS's constants, which every sheet edge of an openEMS file must use to
# reproduce its results. c is the measured (1/l_1 + 17/l_2)/4 (unused: the
# capacitance is formed from l_1 and l_2).
TABLE = np.array([
    [0.137084340054, 0.02222457325, 0.119282088951, 1.302754546, 0.0990690603255, 10.62245057],
    [0.124432770979, 0.019525936, 0.117650643055, 1.2992612, 0.0865774432243, 10.219529],
    [0.10874259256, 0.016475925, 0.112495689579, 1.3200334, 0.0726839782207, 10.247559],
    [0.0921545029514, 0.013604945, 0.102373790897, 1.4182922, 0.0598080542444, 10.991476],
    [0.0763924952568, 0.011153572, 0.0877535678803, 1.6743265, 0.0489583437563, 12.704509],
    [0.0623920685841, 0.0091246982, 0.0714852202949, 2.1387697, 0.0400582737111, 15.598306],
    [0.0506870193634, 0.0074560144, 0.0572157790471, 2.7691268, 0.0327551749758, 19.55715],
    [0.0412416168046, 0.0060890102, 0.0461128464864, 3.4988017, 0.026761739013, 24.325811],
    [0.0336492594616, 0.004971778, 0.0375513332623, 4.311448, 0.0218534019281, 29.887339],
    [0.0274825647083, 0.0040593582, 0.030693935758, 5.2662049, 0.017842192351, 36.556805],
    [0.0224415656409, 0.0033144285, 0.0250704153117, 6.4439781, 0.0145678049496, 44.753744],
    [0.0183231737407, 0.0027062229, 0.0204687079875, 7.8934045, 0.0118946020796, 54.815747],
    [0.0149608078551, 0.0022096219, 0.0167126250576, 9.6674121, 0.00971190254458, 67.135337],
    [0.0122154505375, 0.0018041488, 0.0136458082892, 11.8401, 0.00792973544699, 82.223603],
    [0.00997387466324, 0.0014730814, 0.0111417587353, 14.501103, 0.00647460224422, 100.7029],
    [0.00814363571331, 0.0012027661, 0.00909721105062, 17.760148, 0.00528649098115, 123.33532],
    [0.0066492519176, 0.0009820545, 0.00742784502358, 21.751641, 0.00431640220756, 151.05424],
    [0.00542909273748, 0.00080184417, 0.00606481357423, 26.640202, 0.00352432807109, 185.00275],
    [0.00443283701916, 0.0006547032, 0.00495190327264, 32.627421, 0.00287760227497, 226.58098],
    [0.00361939779282, 0.00053456309, 0.0040432162758, 39.960208, 0.00234955292005, 277.50354],
    [0.00295522765367, 0.00043646901, 0.00330127701783, 48.941, 0.00191840249878, 339.87044],
    [0.00241293536167, 0.0003563757, 0.00269548714004, 59.940125, 0.00156636976862, 416.2535],
    [0.00197015616651, 0.00029097973, 0.00220086344996, 73.411114, 0.00127893644741, 509.8022],
    [0.00160862981206, 0.00023758431, 0.00179700862248, 89.909314, 0.00104424855814, 624.37284],
    [0.0013134233954, 0.00019398532, 0.00146720336246, 110.11961, 0.000852619746587, 764.72806],
    [0.00107242246864, 0.00015838974, 0.0011980129395, 134.86311, 0.000696166544835, 936.55255],
    [0.000903138344057, 0.00012996173, 0.00109385610511, 149.27697, 0.000569245491525, 1000.0],
    [0.000767497363702, 0.00010602016, 0.00106846334836, 153.52594, 0.000462047579022, 1000.0],
    [0.000648257956771, 8.5842202e-05, 0.00106765935995, 148.93717, 0.000372313090849, 1000.0],
    [0.000545069956667, 6.9225859e-05, 0.00110017492041, 119.35233, 0.000298911971364, 1000.0],
], dtype=np.float64)


def _r32(x: float) -> float:
    return float(np.float32(x))


def sheet_frequency(signal, f_max: float | None) -> float:
    """The frequency the sheet model is chosen for (sheet_frequency,
    src/compile/openems_sheet.rs:172-181): f0 + fc of a Gaussian, f0 of a
    sine, else the file's f_max (0 without one)."""
    if signal.kind == 0:
        return signal.f0 + signal.fc
    if signal.kind == 1:
        return signal.f0
    return f_max or 0.0


def bin_index(sigma: float, t: float, f: float) -> int:
    """The bin of a sheet of conductivity sigma [S/m] and thickness t [m] at
    frequency f [Hz] with openEMS's f32 steps (bin, src/compile/
    openems_sheet.rs:183-205): G = f32(σt), X = f32(8/(G·μ0·t)),
    (t/δ)² = f32(4·f32(2πf)/X), ν = (t/δ)²/80; 0 below ν = 1, then
    ⌊log_1.5 ν⌋ + 1, at most 29."""
    t = _r32(t)
    g = _r32(_r32(sigma) * t)
    x = _r32(8.0 / (g * OPENEMS_MU0 * t))
    w = _r32(2.0 * math.pi * f)
    nu = _r32(4.0 * w / x) / 80.0
    if math.isnan(nu) or nu < 1.0:
        return 0
    k = math.floor(math.log10(nu) / math.log10(1.5)) + 1.0
    return 29 if k >= 29.0 else int(k)


def edge_circuit(sigma: float, t: float, l_over_w: float, row) -> tuple[list[tuple[float, float]], float, float]:
    """(branches [(L, R)] × 2, C/dt², G) of a sheet edge with l/w the edge
    length over the sheet width, bin row `row`, with openEMS's f32 steps
    (edge_circuit, src/compile/openems_sheet.rs:219-243): per square
    L_b = f32(l_b·8/(G·X)), R_b = f32(r_b/G), G_s = f32(g·G); per edge with
    k = f32(l/w): L = f32(L_b·k), R = f32(R_b·k), G_e = f32(G_s/k),
    C/dt² = f32(1/L_1)/4 + f32(1/L_2)/4 + 4/L_2."""
    t = _r32(t)
    g = _r32(_r32(sigma) * t)
    x = _r32(8.0 / (g * OPENEMS_MU0 * t))
    q = 8.0 / (g * x)
    k = _r32(l_over_w)
    branches = [(_r32(_r32(lb * q) * k), _r32(_r32(rb / g) * k)) for lb, rb in ((row[2], row[3]), (row[4], row[5]))]
    l1, l2 = branches[0][0], branches[1][0]
    c_per_dt2 = _r32(1.0 / l1) / 4.0 + _r32(1.0 / l2) / 4.0 + 4.0 / l2
    return branches, c_per_dt2, _r32(_r32(row[0] * g) / k)
