"""The host library's set-up arithmetic against the reference's closed-form
unit tests of the coefficients (src/engine/coeffs.rs:1088-1202), called on
libems_host.so directly: the oracle consumes what this library builds, so
these checks pin the shared set-up without going through the oracle.

* the Courant limit and the time-step rules (coeffs.rs:1088-1107);
* the area-weighted parallel permittivity and conductivity of an E edge
  between a dielectric and vacuum, and of a corner edge (coeffs.rs:1109-1137);
* the series permeability and magnetic loss of a dual edge across two half
  cells, a homogeneous one and a boundary one (coeffs.rs:1139-1161);
* PEC faces, PEC edges, padding, the loss coefficients and a PMC face's
  half dual face (coeffs.rs:1163-1201).

CPU only.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import ems_b200 as E

C0, EPS0, MU0 = E.c0(), E.eps0(), E.mu0()


def rel(a, b):
    return abs((a - b) / b)


def test_courant_limit_and_time_step_rules():
    m = E.Model.uniform([4, 4, 4], [1e-3, 2e-3, 1e-3])
    lim = m.courant_limit
    want = 1.0 / (C0 * math.sqrt(1e6 + 0.25e6 + 1e6))
    assert rel(lim, want) < 1e-14
    m.build()
    assert rel(m.dt, 0.99 * want) < 1e-14
    for dt, ok in [(0.5 * lim, True), (lim, True), (1.0001 * lim, False), (-1.0, False), (float("nan"), False)]:
        mm = E.Model.uniform([4, 4, 4], [1e-3, 2e-3, 1e-3])
        if ok:
            mm.build(dt=dt)
            assert mm.dt == dt
        else:
            with pytest.raises(Exception):
                mm.build(dt=dt)
    for s in (1.01, 0.0):
        with pytest.raises(Exception):
            E.Model.uniform([4, 4, 4], [1e-3, 2e-3, 1e-3]).build(courant=s)
    # A graded grid uses the smallest cell.
    g2 = E.Model([0.0, 1.0, 1.5], [0.0, 1.0], [0.0, 1.0])
    assert rel(g2.courant_limit, 1.0 / (C0 * math.sqrt(4.0 + 1.0 + 1.0))) < 1e-14


def test_edge_between_dielectric_and_vacuum():
    """2 × 2 × 2 cells, non-uniform in y and z; the y < 1 half (cells j = 0)
    ε_r = 4, κ = 2. The x edge at node (0, 1, 1) has the dual face
    y ∈ [0.5, 2], z ∈ [1, 2.5]: dielectric area 0.5·1.5, vacuum 1·1.5."""
    m = E.Model([0.0, 1.0, 2.0], [0.0, 1.0, 3.0], [0.0, 2.0, 3.0])
    m.fill(m.cells().box([0, 0, 0], [2, 1, 2]), m.material(eps_r=4.0, kappa=2.0))
    m.build()
    eps, kappa = m.edge_material(0, E.X, (0, 1, 1))
    a_diel, a_vac = 0.5 * (1.0 + 0.5), 1.0 * (1.0 + 0.5)
    area = a_diel + a_vac
    # C = ε0·(4·a_diel + a_vac)/l and G = 2·a_diel/l with l = 1: the
    # effective ε_r and κ are the area-weighted means.
    assert rel(EPS0 * eps * area, EPS0 * (4.0 * a_diel + a_vac)) < 1e-14
    assert rel(kappa * area, 2.0 * a_diel) < 1e-14
    assert rel(eps, (4.0 * a_diel + a_vac) / area) < 1e-14
    # The corner edge at the domain edge: a single quarter cell, ε_r = 4.
    eps_c, _ = m.edge_material(0, E.X, (1, 0, 0))
    assert rel(eps_c, 4.0) < 1e-14


def test_dual_edge_series():
    """x dual edge through node 1 of lines x = 0, 1, 3: half cells of 0.5
    (vacuum) and 1.0 (μ_r 3, σ_m 5), area 2. L is the series combination,
    R = L²·(σ_m·A/l₂)/L₂²."""
    m = E.Model([0.0, 1.0, 3.0], [0.0, 1.0], [0.0, 2.0])
    m.fill(m.cells().box([1, 0, 0], [2, 1, 1]), m.material(mu_r=3.0, sigma_m=5.0))
    m.build()
    mu, sig = m.edge_material(1, E.X, (1, 0, 0))
    area, l_star = 2.0, 1.5
    l1, l2 = MU0 * area / 0.5, MU0 * 3.0 * area / 1.0
    want = 1.0 / (1.0 / l1 + 1.0 / l2)
    assert rel(MU0 * mu * area / l_star, want) < 1e-14
    assert rel(sig * area / l_star, want * want * (5.0 * area / 1.0) / (l2 * l2)) < 1e-14
    # A homogeneous dual edge: L = μ·A/l*, R = σ·A/l*; a boundary one: one half cell.
    m2 = E.Model([0.0, 1.0, 3.0], [0.0, 1.0], [0.0, 2.0])
    m2.fill(m2.cells().box([0, 0, 0], [2, 1, 1]), m2.material(mu_r=2.0, sigma_m=7.0))
    m2.build()
    mu, sig = m2.edge_material(1, E.X, (1, 0, 0))
    assert rel(MU0 * mu * area / 1.5, MU0 * 2.0 * area / 1.5) < 1e-14
    assert rel(sig * area / 1.5, 7.0 * area / 1.5) < 1e-14
    mu, _ = m2.edge_material(1, E.X, (2, 0, 0))
    assert rel(MU0 * mu * area / 1.0, MU0 * 2.0 * area / 1.0) < 1e-14


def _lossy_cube(faces):
    m = E.Model.uniform([3, 3, 3], [1e-3] * 3)
    m.fill(m.cells().box([0, 0, 0], [3, 3, 3]), m.material(kappa=1.0))
    m.pec_edges(E.Z, [1, 1, 1], [1, 1, 1])
    m.faces(faces)
    m.build()
    return m


def test_faces_pec_and_loss():
    m = _lossy_cube([E.PEC] * 6)
    dt = m.dt
    ca = [m.coeff(a) for a in range(3)]
    cb = [m.coeff(3 + a) for a in range(3)]
    db = [m.coeff(9 + a) for a in range(3)]
    # A tangential edge on the x_min face is PEC; the interior one is not.
    assert cb[E.Y][0, 1, 1] == 0.0
    assert cb[E.Y][1, 1, 1] > 0.0
    # The PEC edge.
    assert cb[E.Z][1, 1, 1] == 0.0 and ca[E.Z][1, 1, 1] == 0.0
    # The normal edge touching the face is not tangential.
    assert cb[E.X][0, 1, 1] > 0.0
    # Padding.
    assert cb[E.X][3, 1, 1] == 0.0
    assert db[E.X][1, 3, 1] == 0.0
    # Loss coefficients of the interior x edge: C = ε0·A/l, G = κ·A/l.
    c, g = EPS0 * 1e-3, 1.0 * 1e-3
    want = (c - g * dt / 2.0) / (c + g * dt / 2.0)
    assert rel(float(ca[E.X][1, 1, 1]), want) < 1e-6
    assert want < 1.0
    cap = dt * (1.0 + float(ca[E.X][1, 1, 1])) / (2.0 * float(cb[E.X][1, 1, 1]))
    assert rel(cap, c) < 1e-6
    # PMC on x_min keeps the face edges alive with half the dual face.
    p = _lossy_cube([E.PMC] + [E.PEC] * 5)
    cbp = p.coeff(3 + E.Y)
    cap_face = dt * (1.0 + float(p.coeff(E.Y)[0, 1, 1])) / (2.0 * float(cbp[0, 1, 1]))
    assert rel(cap_face, 0.5 * c) < 1e-6
    assert cbp[0, 1, 1] > 0.0
    # But not where the x_min face meets the PEC z_min face.
    assert cbp[0, 1, 0] == 0.0
