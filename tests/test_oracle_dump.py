"""Field samplers (src/engine/dump.rs FieldSampler) on the host and the
oracle, against the reference's dump tests (tests/dump.rs:17-265, 491-546)
and closed forms of the derived quantities.

* Node values: E interpolated along its own axis, H across its two
  transverse axes, on a non-uniform grid with analytic linear fields; the
  outer nodes take the adjacent cell midpoint (dump.rs:138-161).
* Cell centres: exact for linear fields (dump.rs:164-196); a degenerate
  cell-centre plane uses the node rule (199-219); sub-sampling and a single
  point (222-255); a box outside the grid is refused (258-265).
* Derived quantities: D = ε·E, J = κ·E, B = μ·H in a uniform medium (the
  effective edge values the coefficients hold), rot H of a linear H field
  its constant curl at the interior edges.
* The same samples for any oracle thread count (dump.rs:518-546).

CPU only.
"""
from __future__ import annotations

import numpy as np
import pytest

import ems_b200 as E
from oracle import OracleEngine

MM = 1e-3
LINES = (np.array([0.0, 1.0, 2.5, 4.5, 5.0]) * MM, np.array([0.0, 0.7, 1.9, 2.4, 3.6]) * MM,
         np.array([0.0, 0.4, 1.0, 2.2]) * MM)


def e_field(a, p):
    x, y, z = p
    return (2.0 + 3.0 * x + 5.0 * y, 1.0 - 2.0 * y + 4.0 * z, 3.0 + x + z)[a]


def h_field(a, p):
    x, y, z = p
    return (1.0 + 2.0 * y + 3.0 * z, 2.0 - x + z, x + 2.0 * y)[a]


def mm(a, i):
    return LINES[a][i] / MM


def mid_mm(a, i):
    return 0.5 * (LINES[a][i] + LINES[a][i + 1]) / MM


def delta(a, i):
    return LINES[a][i + 1] - LINES[a][i]


def dual_delta(a, i):
    n = len(LINES[a])
    lo = delta(a, i - 1) if i > 0 else 0.0
    hi = delta(a, i) if i + 1 < n else 0.0
    return 0.5 * (lo + hi)


def analytic_model(material=None):
    m = E.Model(*LINES)
    if material is not None:
        m.fill(m.cells().box([0, 0, 0], [4, 4, 3]), m.material(**material))
        m.faces([E.PMC] * 6)  # no PEC face edges: every edge keeps its material
    m.build()
    return m


def set_analytic(o, m):
    """tests/dump.rs:62-90: u, i the integral form of the analytic fields."""
    n = m.nodes
    u = [np.zeros(n, np.float32) for _ in range(3)]
    i = [np.zeros(n, np.float32) for _ in range(3)]
    for node in np.ndindex(*n):
        for a in range(3):
            if node[a] + 1 < n[a]:
                p = [mm(b, node[b]) for b in range(3)]
                p[a] = mid_mm(a, node[a])
                u[a][node] = np.float32(e_field(a, p) * delta(a, node[a]))
            b, c = (a + 1) % 3, (a + 2) % 3
            if node[b] + 1 < n[b] and node[c] + 1 < n[c]:
                p = [0.0] * 3
                p[a] = mm(a, node[a])
                p[b] = mid_mm(b, node[b])
                p[c] = mid_mm(c, node[c])
                i[a][node] = np.float32(h_field(a, p) * dual_delta(a, node[a]))
    for a in range(3):
        o.set_field(0, a, u[a])
        o.set_field(1, a, i[a])


def node_rule_pos(q, a, node, n):
    """tests/dump.rs:99-114: where the node rule evaluates component a."""
    out = []
    for b in range(3):
        i = node[b]
        interp = (a != b) if q == E.DUMP_H else (a == b)
        if interp and i == 0:
            out.append(mid_mm(b, 0))
        elif interp and i == n[b] - 1:
            out.append(mid_mm(b, n[b] - 2))
        else:
            out.append(mm(b, i))
    return out


def close(got, want, what):
    got = float(np.float32(got))
    assert abs(got - want) <= 2e-6 * max(abs(want), 1.0), (what, got, want)


@pytest.fixture(scope="module")
def analytic():
    m = analytic_model()
    o = OracleEngine(m, threads=1)
    set_analytic(o, m)
    return m, o


def test_node_values_are_converted_and_interpolated(analytic):
    m, o = analytic
    n = m.nodes
    for q, fn in ((E.DUMP_E, e_field), (E.DUMP_H, h_field)):
        s = E.Sampler(m, q, E.NODES)
        assert s.dims == n
        v = o.sample(s).reshape(*n, 3)
        for node in np.ndindex(*n):
            for a in range(3):
                close(v[node][a], fn(a, node_rule_pos(q, a, node, n)), (q, a, node))


def test_cell_centre_values_are_exact_for_linear_fields(analytic):
    m, o = analytic
    c = tuple(x - 1 for x in m.nodes)
    for q, fn in ((E.DUMP_E, e_field), (E.DUMP_H, h_field)):
        s = E.Sampler(m, q, E.CELL_CENTERS)
        assert s.dims == c
        assert np.array_equal(s.coords[0], 0.5 * (LINES[0][1:] + LINES[0][:-1]))
        v = o.sample(s).reshape(*c, 3)
        for cell in np.ndindex(*c):
            p = [mid_mm(b, cell[b]) for b in range(3)]
            for a in range(3):
                close(v[cell][a], fn(a, p), (q, a, cell))


def test_degenerate_cell_centre_plane_uses_node_rule(analytic):
    m, o = analytic
    s = E.Sampler(m, E.DUMP_E, E.CELL_CENTERS, [4, 2, 0], [0, 2, 3])  # corners in any order
    assert s.dims == (4, 1, 3)
    assert list(s.coords[1]) == [LINES[1][2]]
    v = o.sample(s).reshape(4, 1, 3, 3)
    for i in range(4):
        for k in range(3):
            p = [mid_mm(0, i), mm(1, 2), mid_mm(2, k)]
            for a in range(3):
                close(v[i, 0, k, a], e_field(a, p), "plane")


def test_sub_sampling_and_a_single_point(analytic):
    m, o = analytic
    full = o.sample(E.Sampler(m, E.DUMP_H, E.NODES)).reshape(*m.nodes, 3)
    s = E.Sampler(m, E.DUMP_H, E.NODES, [1, 0, 0], [4, 4, 3], stride=[2, 1, 3])
    assert s.dims == (2, 5, 2)
    assert list(s.coords[0]) == [LINES[0][1], LINES[0][3]]
    assert list(s.coords[2]) == [LINES[2][0], LINES[2][3]]
    sub = o.sample(s).reshape(2, 5, 2, 3)
    assert np.array_equal(sub, full[[1, 3]][:, :, [0, 3]])
    s1 = E.Sampler(m, E.DUMP_E, E.NODES, [2, 3, 1], [2, 3, 1])
    assert s1.dims == (1, 1, 1) and len(s1) == 1


def test_region_must_fit():
    m = analytic_model()
    with pytest.raises(ValueError):
        E.Sampler(m, E.DUMP_E, E.NODES, [0, 0, 0], [4, 5, 3])


def test_native_positions_are_raw_edge_values(analytic):
    m, o = analytic
    n = m.nodes
    u = [o.field(0, a) for a in range(3)]
    i = [o.field(1, a) for a in range(3)]
    e = o.sample(E.Sampler(m, E.DUMP_E, E.NATIVE)).reshape(*n, 3)
    h = o.sample(E.Sampler(m, E.DUMP_H, E.NATIVE)).reshape(*n, 3)
    s = E.Sampler(m, E.DUMP_H, E.NATIVE)
    assert np.allclose(s.coords[0][:-1], 0.5 * (LINES[0][1:] + LINES[0][:-1]))
    for node in np.ndindex(*n):
        for a in range(3):
            want_e = (1.0 / delta(a, node[a])) * float(u[a][node]) if node[a] + 1 < n[a] else 0.0
            assert e[node][a] == want_e
            assert h[node][a] == (1.0 / dual_delta(a, node[a])) * float(i[a][node])


def test_derived_quantities_in_a_uniform_medium():
    """D = ε0·ε_r·E, J = κ·E, B = μ0·μ_r·H at the cell centres, PMC faces.
    The material factors come from the f32 coefficients: D and B agree to
    ~1e-6; G = (1 − ca)/cb loses digits to ca near 1 (1e-5)."""
    eps_r, kappa, mu_r = 3.0, 0.25, 2.0
    m = analytic_model(dict(eps_r=eps_r, kappa=kappa, mu_r=mu_r))
    o = OracleEngine(m, threads=1)
    set_analytic(o, m)
    e = o.sample(E.Sampler(m, E.DUMP_E, E.CELL_CENTERS))
    h = o.sample(E.Sampler(m, E.DUMP_H, E.CELL_CENTERS))
    d = o.sample(E.Sampler(m, E.DUMP_D, E.CELL_CENTERS))
    j = o.sample(E.Sampler(m, E.DUMP_J, E.CELL_CENTERS))
    b = o.sample(E.Sampler(m, E.DUMP_B, E.CELL_CENTERS))
    np.testing.assert_allclose(d, E.eps0() * eps_r * e, rtol=2e-6)
    np.testing.assert_allclose(j, kappa * e, rtol=1e-5)
    np.testing.assert_allclose(b, E.mu0() * mu_r * h, rtol=2e-6)


def test_rot_h_of_a_linear_field_is_its_curl(analytic):
    """H = (1 + 2y + 3z, 2 − x + z, x + 2y) (mm): ∇×H = (1, 2, −3) per mm.
    The circulation over a dual face of interior edges is exact."""
    m, o = analytic
    s = E.Sampler(m, E.DUMP_ROTH, E.NATIVE)
    v = o.sample(s).reshape(*m.nodes, 3)
    want = np.array([1.0, 2.0, -3.0]) / MM
    n = m.nodes
    checked = 0
    for node in np.ndindex(*n):
        for a in range(3):
            b, c = (a + 1) % 3, (a + 2) % 3
            if node[a] + 1 < n[a] and 0 < node[b] < n[b] - 1 and 0 < node[c] < n[c] - 1:
                assert abs(v[node][a] - want[a]) <= 2e-5 * abs(want[a]), (node, a, v[node][a])
                checked += 1
    assert checked > 10


def test_openems_sampler_rules(analytic):
    """FieldSampler::openems: H at a node is the plain mean of the four
    dual edges around it, 0 on the outer nodes."""
    m, o = analytic
    n = m.nodes
    s = E.Sampler(m, E.DUMP_H, E.NODES, indices=[range(n[0]), range(n[1]), range(n[2])])
    v = o.sample(s).reshape(*n, 3)
    i = [o.field(1, a) for a in range(3)]
    for node in np.ndindex(*n):
        a = 0
        if 0 < node[1] < n[1] - 1 and 0 < node[2] < n[2] - 1:
            x, y, z = node
            w = 1.0 / dual_delta(0, x)
            want = 0.0
            for (jj, wy) in ((y - 1, 0.5), (y, 0.5)):
                for (kk, wz) in ((z - 1, 0.5), (z, 0.5)):
                    want += w * wy * wz * 1.0 * float(i[0][x, jj, kk])
            assert v[node][a] == want
        elif node[1] in (0, n[1] - 1) or node[2] in (0, n[2] - 1):
            assert v[node][a] == 0.0
    with pytest.raises(ValueError):
        E.Sampler(m, E.DUMP_H, E.NODES, indices=[[0, 0], [1], [1]])


def test_samples_do_not_depend_on_threads():
    """tests/dump.rs:518-546: a scrambled state, run 60 steps."""
    def lines(n, s):
        return np.array([s * (i + 0.15 * np.sin(i)) for i in range(n)])

    def run(threads):
        m = E.Model(lines(12, 1e-3), lines(10, 1.2e-3), lines(8, 0.9e-3))
        m.build()
        o = OracleEngine(m, threads=threads)
        rng = np.random.default_rng(7)
        n = m.nodes
        for a in range(3):
            x = ((rng.random(n) - 0.5) * 1e-3).astype(np.float32)
            b, c = (a + 1) % 3, (a + 2) % 3
            ok = np.zeros(n, bool)
            ok[tuple(slice(None, -1) if t == a else slice(1, -1) for t in range(3))] = True
            o.set_field(0, a, np.where(ok, x, 0).astype(np.float32))
        o.run(60)
        return (o.sample(E.Sampler(m, E.DUMP_E, E.NODES, stride=[1, 2, 1])),
                o.sample(E.Sampler(m, E.DUMP_H, E.CELL_CENTERS)),
                o.sample(E.Sampler(m, E.DUMP_ROTH, E.CELL_CENTERS)))

    r1, r4 = run(1), run(4)
    assert any(np.any(x != 0) for x in r1)
    for a, b in zip(r1, r4):
        assert np.array_equal(a, b)
