"""Seeded synthetic models of the benchmark configurations.

No model files or datasets are used: every model is built from a fixed seed
with the shapes, sizes and value ranges of the configuration it stands for.

* :func:`vacuum_box` — a vacuum box of uniform cells with CPML on all six
  faces, a soft E_z point source at the centre edge (Gaussian f0, fc) and
  E_z point probes at seeded interior edges (100³ cells, 1 mm, CPML 8,
  2 GHz / 1 GHz, 4 probes for the small plain-method configuration).
* :func:`dispersive_box` — a uniform box with CPML, a centred sphere of a
  two-pole Lorentz medium (ε∞ 2.0, plasma 5 and 8 GHz, resonance 3 and
  6 GHz, damping 0.1–0.3 GHz from the seed), a Drude slab (plasma 10 GHz,
  collision 1 GHz) normal to z, and a soft E_x sheet source (512³ cells,
  0.5 mm, CPML 10, sphere radius 80 cells, slab 20 cells for the large
  configuration). Pole frequencies enter as angular frequencies
  ω = 2π·f (engine-level ``Pole`` convention, src/engine/dispersive.rs:211-244).
* :func:`patch_antenna` — a graded-mesh patch antenna: FR-4 slab on a PEC
  z_min ground, PEC patch, 50 Ω lumped port along z, CPML on the other
  five faces (about 200×200×80 cells for the full configuration).
* :func:`sweep_variant` — one seeded patch variant of the batched sweep on
  its own graded N × N × N mesh (N in 60…160).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

import ems_b200 as E

TWO_PI = 2.0 * math.pi


@dataclass
class Workload:
    """A built model and what the runs need to know about it."""

    name: str
    model: E.Model
    steps: int
    probes: list[int] = field(default_factory=list)
    port: int | None = None
    source: int | None = None
    info: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        n = self.model.nodes
        return (n[0] - 1) * (n[1] - 1) * (n[2] - 1)


def vacuum_box(n: int = 100, cell: float = 1e-3, cpml: int = 8, steps: int = 2000, f0: float = 2e9,
               fc: float = 1e9, n_probes: int = 4, seed: int = 0x5EED, courant: float = 0.99) -> Workload:
    m = E.Model.uniform([n, n, n], [cell] * 3)
    m.build(courant=courant)
    if cpml:
        m.add_cpml([cpml] * 6)
    c = n // 2
    src = m.add_source(E.SOFT_E, [(E.Z, (c, c, c), 1.0)], f0, fc, steps)
    rng = np.random.default_rng(seed)
    lo, hi = cpml + 1, n - cpml - 1
    probes = []
    for _ in range(n_probes):
        node = tuple(int(v) for v in rng.integers(lo, hi, size=3))
        probes.append(m.add_probe(E.VOLTAGE, [(E.Z, node, 1.0)]))
    return Workload(f"vacuum_box_{n}", m, steps, probes, source=src,
                    info={"cells": n, "cell_m": cell, "cpml": cpml, "f0": f0, "fc": fc, "courant": courant})


def lorentz_poles(seed: int) -> list[E.Pole]:
    rng = np.random.default_rng(seed)
    gam = rng.uniform(0.1e9, 0.3e9, size=2)
    return [E.Pole.lorentz(TWO_PI * 5e9, TWO_PI * 3e9, TWO_PI * gam[0]),
            E.Pole.lorentz(TWO_PI * 8e9, TWO_PI * 6e9, TWO_PI * gam[1])]


def dispersive_box(n: int = 512, cell: float = 0.5e-3, cpml: int = 10, radius: float = 80.0, slab: int = 20,
                   steps: int = 4000, scheme: int = E.LEAPFROG, seed: int = 0x5EED, f0: float = 5e9,
                   fc: float = 3e9, courant: float = 0.99, probes: bool = True) -> Workload:
    m = E.Model.uniform([n, n, n], [cell] * 3)
    sphere = m.cells().sphere([n / 2, n / 2, n / 2], radius)
    m.fill(sphere, m.material(eps_r=2.0))
    m.build(courant=courant)
    if cpml:
        m.add_cpml([cpml] * 6)
    d = E.Dispersive()
    d.fill_cells(m, sphere, lorentz_poles(seed))
    # The Drude slab normal to z, beyond the sphere, across the whole x-y extent.
    z0 = int(round(n * 0.80))
    slab_cells = m.cells().box([0, 0, z0], [n, n, min(n, z0 + slab)])
    d.fill_cells(m, slab_cells, [E.Pole.drude(TWO_PI * 10e9, TWO_PI * 1e9)])
    m.add_dispersive(d, scheme)
    # Soft E_x sheet on the plane z = zs over the interior (outside the CPML).
    zs = cpml + max(2, n // 10)
    ii, jj = np.meshgrid(np.arange(cpml, n - cpml), np.arange(cpml, n + 1 - cpml), indexing="ij")
    nodes = np.stack([ii.ravel(), jj.ravel(), np.full(ii.size, zs)], axis=1)
    src = m.add_source_arrays(E.SOFT_E, np.zeros(len(nodes), np.int32), nodes, np.ones(len(nodes)), f0, fc, steps)
    pr = []
    if probes:
        c = n // 2
        for node in [(c, c, c), (c, c, zs + (c - zs) // 2), (c, c, z0 + slab + 2), (c // 2, c, c)]:
            pr.append(m.add_probe(E.VOLTAGE, [(E.X, node, 1.0)]))
        pr.append(m.add_probe(E.CURRENT, [(E.Y, (c, c, c), 1.0)]))
    return Workload(f"dispersive_box_{n}", m, steps, pr, source=src,
                    info={"cells": n, "cell_m": cell, "cpml": cpml, "radius": radius, "slab": slab,
                          "scheme": "leapfrog" if scheme == E.LEAPFROG else "trapezoidal", "f0": f0, "fc": fc,
                          "sheet_edges": int(len(nodes)), "courant": courant})


def graded_lines(length: float, fine: float, coarse: float, fine_regions: list[tuple[float, float]],
                 grow: float, rng: np.random.Generator, jitter: float) -> np.ndarray:
    """Mesh lines 0..length: cells of size ``fine`` inside ``fine_regions``,
    growing by ``grow`` per cell away from them up to ``coarse``, each cell
    scaled by a seeded factor in [1 − jitter, 1 + jitter] (at most ``coarse``)."""
    lines = [0.0]
    x = 0.0
    while x < length - 1e-12:
        dist = min((0.0 if a <= x <= b else min(abs(x - a), abs(x - b))) for a, b in fine_regions)
        h = min(coarse, fine * grow ** (dist / fine)) if dist > 0 else fine
        h = min(coarse, h * (1.0 + jitter * (2.0 * rng.random() - 1.0)))
        x = min(length, x + h)
        if length - x < 0.3 * fine:
            x = length
        lines.append(x)
    return np.array(lines)


def patch_antenna(scale: float = 1.0, seed: int = 0x5EED, steps: int = 30000, cpml: int = 8,
                  courant: float = 0.99) -> Workload:
    """Patch antenna on a graded mesh (scale 1.0: about 200×200×80 cells)."""
    mm = 1e-3
    rng = np.random.default_rng(seed)
    sub = 60.0 * mm
    patch = 28.0 * mm
    h = 1.6 * mm
    air = 30.0 * mm * scale
    lx = sub + 2 * air
    c = lx / 2
    fine, coarse = 0.25 * mm / scale, 1.0 * mm / scale
    edges = [(c - patch / 2 - 1 * mm, c - patch / 2 + 1 * mm), (c + patch / 2 - 1 * mm, c + patch / 2 + 1 * mm),
             (c - sub / 2 - 0.5 * mm, c - sub / 2 + 0.5 * mm), (c + sub / 2 - 0.5 * mm, c + sub / 2 + 0.5 * mm),
             (c + 8 * mm - 0.5 * mm, c + 8 * mm + 0.5 * mm)]
    xl = graded_lines(lx, fine, coarse, edges, 1.08, rng, 0.1)
    yl = graded_lines(lx, fine, coarse, edges[:4] + [(c - 0.5 * mm, c + 0.5 * mm)], 1.08, rng, 0.1)
    lz = h + 62.0 * mm * scale
    zl_sub = np.linspace(0.0, h, 8)
    zl_air = graded_lines(lz - h, fine, coarse, [(0.0, 0.5 * mm)], 1.1, rng, 0.1) + h
    zl = np.concatenate([zl_sub, zl_air[1:]])
    m = E.Model(xl, yl, zl)
    near = lambda lines, v: int(np.argmin(np.abs(lines - v)))  # noqa: E731
    i0, i1 = near(xl, c - sub / 2), near(xl, c + sub / 2)
    j0, j1 = near(yl, c - sub / 2), near(yl, c + sub / 2)
    kh = len(zl_sub) - 1
    m.fill(m.cells().box([i0, j0, 0], [i1, j1, kh]), m.material(eps_r=4.3))
    pi0, pi1 = near(xl, c - patch / 2), near(xl, c + patch / 2)
    pj0, pj1 = near(yl, c - patch / 2), near(yl, c + patch / 2)
    m.pec_edges(E.X, [pi0, pj0, kh], [pi1 - 1, pj1, kh])
    m.pec_edges(E.Y, [pi0, pj0, kh], [pi1, pj1 - 1, kh])
    m.faces([E.PEC] * 6)
    m.build(courant=courant)
    m.add_cpml([cpml, cpml, cpml, cpml, 0, cpml])
    px, py = near(xl, c + 8 * mm), near(yl, c)
    port = m.add_lumped_port(E.Z, [px, py, 0], [px, py, kh], 50.0, 2e9, 1e9, 1.0, steps)
    n = m.nodes
    return Workload(f"patch_antenna_{n[0] - 1}x{n[1] - 1}x{n[2] - 1}", m, steps, port=port,
                    info={"nodes": n, "port_node": (px, py), "substrate_cells": kh, "courant": courant})


def patch_variant(seed: int, cells: tuple[int, int] = (60, 160), steps: int = 60000, cpml: int = 8,
                  courant: float = 0.99) -> Workload:
    """One seeded patch-antenna variant of the batched sweep: patch side
    8–30 mm, substrate ε_r 2.2–10.2 and thickness 0.8–3.2 mm, port offset
    2–10 mm from the patch centre, PEC ground at z_min, CPML on the other
    five faces, 50 Ω port with a Gaussian f0 = 2 GHz, fc = 1.5 GHz; meshed to
    its own size, N × N × N/2 cells with N drawn from `cells` (graded in z:
    the substrate finer than the air)."""
    mm = 1e-3
    rng = np.random.default_rng(seed)
    side = rng.uniform(8.0, 30.0) * mm
    eps = rng.uniform(2.2, 10.2)
    h = rng.uniform(0.8, 3.2) * mm
    off = rng.uniform(2.0, 10.0) * mm
    n = int(rng.integers(cells[0], cells[1] + 1))
    sub = 2.2 * side + 10 * mm
    lx = sub + 2 * 12.0 * mm
    d = lx / n
    xl = np.arange(n + 1) * d
    nz = max(12, n // 2)
    nsub = max(3, min(nz // 4, int(round(h / (0.5 * d)))))
    air = (nz - nsub) * d * 1.2
    zl = np.concatenate([np.linspace(0.0, h, nsub + 1), h + np.linspace(0.0, air, nz - nsub + 1)[1:]])
    m = E.Model(xl, xl, zl)
    c = lx / 2
    near = lambda lines, v: int(np.argmin(np.abs(lines - v)))  # noqa: E731
    i0, i1 = near(xl, c - sub / 2), near(xl, c + sub / 2)
    m.fill(m.cells().box([i0, i0, 0], [i1, i1, nsub]), m.material(eps_r=eps))
    p0, p1 = near(xl, c - side / 2), near(xl, c + side / 2)
    m.pec_edges(E.X, [p0, p0, nsub], [p1 - 1, p1, nsub])
    m.pec_edges(E.Y, [p0, p0, nsub], [p1, p1 - 1, nsub])
    m.faces([E.PEC] * 6)
    m.build(courant=courant)
    m.add_cpml([cpml, cpml, cpml, cpml, 0, cpml])
    px, py = near(xl, c + off), near(xl, c)
    port = m.add_lumped_port(E.Z, [px, py, 0], [px, py, nsub], 50.0, 2e9, 1.5e9, 1.0, steps)
    nn = m.nodes
    return Workload(f"patch_variant_{seed}_{nn[0] - 1}x{nn[1] - 1}x{nn[2] - 1}", m, steps, port=port,
                    info={"seed": seed, "side_mm": side / mm, "eps_r": eps, "h_mm": h / mm, "offset_mm": off / mm,
                          "cells": (nn[0] - 1) * (nn[1] - 1) * (nn[2] - 1), "f0": 2e9, "fc": 1.5e9})


def density_lines(length: float, n: int, fine_at: list[float], ratio: float, width: float) -> np.ndarray:
    """Exactly n cells over [0, length], graded: the cell density is `ratio`
    times higher at the points `fine_at` than far from them (a Gaussian bump
    of half-width `width` around each), the lines placed at the inverse of
    the cumulative density."""
    x = np.linspace(0.0, length, 20001)
    bump = np.zeros_like(x)
    for c in fine_at:
        bump = np.maximum(bump, np.exp(-((x - c) / width) ** 2))
    dens = 1.0 + (ratio - 1.0) * bump
    cum = np.concatenate([[0.0], np.cumsum(0.5 * (dens[1:] + dens[:-1]) * np.diff(x))])
    cum *= n / cum[-1]
    lines = np.interp(np.arange(n + 1, dtype=float), cum, x)
    lines[0], lines[-1] = 0.0, length
    return lines


def sweep_variant(seed: int, cells: tuple[int, int] = (60, 160), steps: int = 60000, cpml: int = 8,
                  courant: float = 0.99) -> Workload:
    """One seeded patch-antenna variant of the batched sweep: patch side
    8–30 mm, substrate ε_r 2.2–10.2 and thickness 0.8–3.2 mm, port offset
    2–10 mm from the patch centre, PEC ground at z_min, CPML on the other
    five faces, 50 Ω port with a Gaussian f0 = 2 GHz, fc = 1.5 GHz; meshed to
    its own size, N × N × N cells with N drawn from `cells`: x and y graded
    three times finer at the patch edges and the port than far from them, z
    with uniform substrate cells below air cells that grow away from it."""
    mm = 1e-3
    rng = np.random.default_rng(seed)
    side = rng.uniform(8.0, 30.0) * mm
    eps = rng.uniform(2.2, 10.2)
    h = rng.uniform(0.8, 3.2) * mm
    off = rng.uniform(2.0, 10.0) * mm
    n = int(rng.integers(cells[0], cells[1] + 1))
    sub = 2.2 * side + 10 * mm
    lx = sub + 2 * 12.0 * mm
    c = lx / 2
    width = max(1.0 * mm, 4.0 * lx / n)
    xl = density_lines(lx, n, [c - side / 2, c + side / 2, c + off], 3.0, width)
    yl = density_lines(lx, n, [c - side / 2, c + side / 2, c], 3.0, width)
    nsub = max(3, min(n // 5, int(round(h / (0.4 * lx / n)))))
    air = 0.8 * lx
    za = density_lines(air, n - nsub, [0.0], 3.0, 3.0 * width)
    zl = np.concatenate([np.linspace(0.0, h, nsub + 1), h + za[1:]])
    m = E.Model(xl, yl, zl)
    near = lambda lines, v: int(np.argmin(np.abs(lines - v)))  # noqa: E731
    i0, i1 = near(xl, c - sub / 2), near(xl, c + sub / 2)
    j0, j1 = near(yl, c - sub / 2), near(yl, c + sub / 2)
    m.fill(m.cells().box([i0, j0, 0], [i1, j1, nsub]), m.material(eps_r=eps))
    p0, p1 = near(xl, c - side / 2), near(xl, c + side / 2)
    q0, q1 = near(yl, c - side / 2), near(yl, c + side / 2)
    m.pec_edges(E.X, [p0, q0, nsub], [p1 - 1, q1, nsub])
    m.pec_edges(E.Y, [p0, q0, nsub], [p1, q1 - 1, nsub])
    m.faces([E.PEC] * 6)
    m.build(courant=courant)
    m.add_cpml([cpml, cpml, cpml, cpml, 0, cpml])
    px, py = near(xl, c + off), near(yl, c)
    port = m.add_lumped_port(E.Z, [px, py, 0], [px, py, nsub], 50.0, 2e9, 1.5e9, 1.0, steps)
    nn = m.nodes
    return Workload(f"sweep_variant_{seed}_{nn[0] - 1}x{nn[1] - 1}x{nn[2] - 1}", m, steps, port=port,
                    info={"seed": seed, "side_mm": side / mm, "eps_r": eps, "h_mm": h / mm, "offset_mm": off / mm,
                          "cells": (nn[0] - 1) * (nn[1] - 1) * (nn[2] - 1), "f0": 2e9, "fc": 1.5e9})
