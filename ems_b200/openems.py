"""openEMS XML models on the engine (a subset of the reference's file path).

Reads an openEMS ``model.xml`` and sets it up the way the reference does
for files (``Simulation::from_xml`` with ``Fdtd::openems_run``; src/sim/
mod.rs:55-190, src/sim/map.rs, src/compile/mod.rs, src/fdtd.rs), runs it on
the CUDA engine (or any engine with the same interface) and writes
openEMS's probe files and excitation signal files (``et``/``ht``).

Restated from the reference:

* the time step: openEMS's criterion (``TimeStepMethod`` 3 Rennings or 1
  Gershgorin, src/engine/timestep.rs), times ``TimeStepFactor``, or
  ``TimeStep``; a sinusoid's period split into whole steps
  (periodic_timestep, timestep.rs:292-296); the run length
  ``NumberOfTimesteps`` cut by ``MaxTime``;
* the coefficients with openEMS's rounding (``CoeffRounding::OpenEms``)
  and magnetic-conductivity average, the curl summed in openEMS's order
  (``CurlOrder::OpenEms``);
* the signals (src/waveform.rs:442-518, src/io/openems/signal.rs):
  openEMS's Gaussian (τ = 3/(2π·fc), delay 3τ, sample 0 zero), sinusoid
  (period repeated), Dirac, step and custom expressions; openEMS's timing
  (src/sim/map.rs:270-307: the field value at time T gets the sample at
  T − dt − ⌊Delay/dt⌋·dt);
* PEC, PMC (openEMS's half-cell PMC, src/compile/mod.rs:1556-1626),
  first-order Mur faces (openEMS's options, the hold of faces that carry an
  E excitation, src/compile/mod.rs:1439-1476) and PML_n layers (openEMS's
  uniaxial layer, src/engine/boundary/upml.rs);
* isotropic or anisotropic materials and metal on box primitives;
  Lorentz, Drude and Debye materials as per-edge leapfrog poles with
  openEMS's edge rule (src/compile/dispersive.rs:1-130);
* E and H excitations (soft, hard) with ``Excite`` and ``Delay``;
* probes (src/sim/map.rs:1150-1380, 1683-1870): voltage along the
  staircase path, current around a loop in the nearest dual plane
  (openEMS's snapping, entry order and f32 sum), native E and H field
  components; openEMS's skip rules; time-domain files every
  ⌊N/OverSampling⌋ steps (N the Nyquist interval), ``FD_Samples`` files,
  H-type files with the sample after the last step;
* the end criterion: openEMS's energy measure checked every Nyquist
  interval and after half a Gaussian's length (src/sim/mod.rs:892-930).

A ``DumpBox`` is read and named in the warnings; openEMS's dump files
(its HDF5/VTK layout) are not written. Refused with ``NotImplementedError``:
cylindrical grids and primitives, plane-wave excitations, curves,
transformations of sources and probes, dispersive media on or beside a Mur
face, lumped elements with inductors or in series on sheets, in PML layers
or under poles, and the other cases named where they are raised.
"""
from __future__ import annotations

import ctypes
import math
import os
import re
import struct
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field

import numpy as np

from . import probe_files as PF

C0 = 299792458.0
TWO_PI = 2.0 * math.pi
FACE_NAMES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")
PEC_FACE, PMC_FACE, MUR_FACE, PML_FACE = 0, 1, 2, 3
MATERIALS = ("Material", "LorentzMaterial", "DebyeMaterial")


# ---------------------------------------------------------------------------
# Custom signal expressions (openEMS's function parser syntax, a subset).

_FUNCS = {"exp": math.exp, "cos": math.cos, "sin": math.sin, "tan": math.tan, "sqrt": math.sqrt,
          "abs": abs, "log": math.log, "log10": math.log10, "atan": math.atan, "cosh": math.cosh,
          "sinh": math.sinh, "tanh": math.tanh}
_TOKEN = re.compile(r"\s*(?:(\d+\.?\d*(?:[eE][-+]?\d+)?|\.\d+(?:[eE][-+]?\d+)?)|([A-Za-z_]\w*)|(<=|>=|!=|.))")


_COMPARE = {"<": lambda a, b: a < b, ">": lambda a, b: a > b, "<=": lambda a, b: a <= b,
            ">=": lambda a, b: a >= b, "=": lambda a, b: a == b, "!=": lambda a, b: a != b}


class Expression:
    """A signal ``f(t)`` or a weighting function ``w(x, y, z)`` in openEMS's
    expression syntax: numbers, the variables named, ``pi``, + − * / ^,
    parentheses, unary minus and the functions of ``_FUNCS`` (parsed once
    into a tree; no evaluation of arbitrary code)."""

    def __init__(self, text: str, variables=("t",)):
        self.text = text
        self.variables = tuple(variables)
        self._tok = [(m.group(1), m.group(2), m.group(3)) for m in _TOKEN.finditer(text) if any(m.groups())]
        self._i = 0
        self._tree = self._compare()
        if self._i != len(self._tok):
            raise ValueError(f"expression {text!r}: unexpected {self._tok[self._i]}")

    def _peek(self):
        return self._tok[self._i] if self._i < len(self._tok) else (None, None, None)

    def _take(self, op):
        if self._peek()[2] == op:
            self._i += 1
            return True
        return False

    def _compare(self):
        """fparser's comparisons (lowest precedence): 1 where true, else 0."""
        node = self._sum()
        while True:
            for op in ("<=", ">=", "!=", "<", ">", "="):
                if self._take(op):
                    node = (op, node, self._sum())
                    break
            else:
                return node

    def _sum(self):
        node = self._product()
        while True:
            if self._take("+"):
                node = ("+", node, self._product())
            elif self._take("-"):
                node = ("-", node, self._product())
            else:
                return node

    def _product(self):
        node = self._unary()
        while True:
            if self._take("*"):
                node = ("*", node, self._unary())
            elif self._take("/"):
                node = ("/", node, self._unary())
            else:
                return node

    def _unary(self):
        if self._take("-"):
            return ("neg", self._unary())
        if self._take("+"):
            return self._unary()
        return self._power()

    def _power(self):
        base = self._atom()
        if self._take("^"):
            return ("^", base, self._unary())
        return base

    def _atom(self):
        num, name, op = self._peek()
        if num is not None:
            self._i += 1
            return ("num", float(num))
        if name is not None:
            self._i += 1
            if name in _FUNCS:
                if not self._take("("):
                    raise ValueError(f"expression {self.text!r}: {name} needs (")
                arg = self._compare()
                if not self._take(")"):
                    raise ValueError(f"expression {self.text!r}: missing )")
                return ("fn", name, arg)
            if name in self.variables:
                return ("var", name)
            if name == "pi":
                return ("num", math.pi)
            raise ValueError(f"expression {self.text!r}: unknown name {name}")
        if self._take("("):
            node = self._compare()
            if not self._take(")"):
                raise ValueError(f"expression {self.text!r}: missing )")
            return node
        raise ValueError(f"expression {self.text!r}: unexpected {op!r}")

    def __call__(self, t: float) -> float:
        def ev(n):
            k = n[0]
            if k == "num":
                return n[1]
            if k == "var":
                return t
            if k == "neg":
                return -ev(n[1])
            if k == "fn":
                return _FUNCS[n[1]](ev(n[2]))
            a, b = ev(n[1]), ev(n[2])
            if k in _COMPARE:
                return 1.0 if _COMPARE[k](a, b) else 0.0
            return {"+": a + b, "-": a - b, "*": a * b, "/": a / b if b != 0 else math.inf}.get(k) \
                if k != "^" else a ** b
        return float(ev(self._tree))

    def evaluate(self, **env):
        """The expression over numpy arrays (or numbers) of its variables."""
        fn = {"exp": np.exp, "cos": np.cos, "sin": np.sin, "tan": np.tan, "sqrt": np.sqrt, "abs": np.abs,
              "log": np.log, "log10": np.log10, "atan": np.arctan, "cosh": np.cosh, "sinh": np.sinh,
              "tanh": np.tanh}

        def ev(n):
            k = n[0]
            if k == "num":
                return n[1]
            if k == "var":
                return np.asarray(env[n[1]], dtype=np.float64)
            if k == "neg":
                return -ev(n[1])
            if k == "fn":
                return fn[n[1]](ev(n[2]))
            a, b = ev(n[1]), ev(n[2])
            if k == "+":
                return a + b
            if k == "-":
                return a - b
            if k == "*":
                return a * b
            if k == "/":
                return np.divide(a, b)
            if k in _COMPARE:
                return np.where(_COMPARE[k](a, b), 1.0, 0.0)
            return np.power(a, b)
        with np.errstate(all="ignore"):
            return np.asarray(ev(self._tree), dtype=np.float64)


# ---------------------------------------------------------------------------
# Signals (src/waveform.rs:442-518).

@dataclass
class Signal:
    """openEMS excitation signal: kind 0 Gaussian (f0, fc), 1 sinusoid
    (f0), 2 Dirac, 3 step, 10 custom expression (f0 for the Nyquist rate)."""

    kind: int
    f0: float = 0.0
    fc: float = 0.0
    expr: Expression | None = None

    @property
    def tau(self) -> float:
        return 3.0 / (TWO_PI * self.fc)

    @property
    def delay(self) -> float:
        return 3.0 * self.tau if self.kind == 0 else 0.0

    def value(self, t: float, dt: float) -> float:
        """Waveform::value with openEMS's sampling convention: sample
        k = ⌊t/dt + ¼⌋ on the E or H grid."""
        k = math.floor(t / dt + 0.25 + 1e-9)
        if self.kind == 0:
            T = self.delay
            if not (k >= 1 and k <= math.floor(2.0 * T / dt + 1e-9)):
                return 0.0
            x = (t - T) / self.tau
            return math.cos(TWO_PI * self.f0 * (t - T)) * math.exp(-x * x)
        if self.kind == 1:
            return math.sin(TWO_PI * self.f0 * t) if (k >= 1 and not self._sine_wrap(dt, k)) else 0.0
        if self.kind == 2:
            return 1.0 if k == 1 else 0.0
        if self.kind == 3:
            return 1.0 if k >= 0 else 0.0
        return self.expr(t)

    def _sine_wrap(self, dt, k):
        p = 1.0 / (self.f0 * dt)
        n = round(p)
        return n >= 1 and abs(p - n) <= 1e-6 * n and (k % n) == 0

    def nyquist_frequency(self):
        if self.kind == 0:
            return self.f0 + self.fc
        if self.kind in (1, 10) and self.f0 > 0:
            return self.f0
        return None

    def nyquist_interval(self, dt: float) -> int:
        f = self.nyquist_frequency()
        if not f or not math.isfinite(f) or f <= 0:
            return 1
        k = math.floor(1.0 / (2.0 * f * dt))
        return int(k) if k >= 1 else 1

    def length(self, dt: float, max_steps: int) -> int:
        """Rows of the ``et``/``ht`` files (src/io/openems/signal.rs:77-104)."""
        if self.kind == 0:
            return min(int(math.floor(2.0 * self.delay / dt)) + 1, max_steps)
        if self.kind == 1:
            return 2 * max(1, round(1.0 / (self.f0 * dt)))
        if self.kind in (2, 3):
            return 2
        return max_steps

    def signal_text(self, dt: float, max_steps: int, offset: float) -> str:
        rows = []
        for k in range(self.length(dt, max_steps)):
            t = (k + offset) * dt
            rows.append(f"{PF.fmt_g(t, 6)}\t{PF.fmt_g(self.value(t, dt), 6)}")
        return "\n".join(rows) + "\n"


# ---------------------------------------------------------------------------
# The file.

@dataclass
class Box:
    p1: tuple
    p2: tuple
    priority: int = 0

    def inside(self, x, y, z, tol):
        """Closed inside test with tolerance ``tol`` (drawing units) over
        broadcastable coordinate arrays."""
        r = True
        for q, v in enumerate((x, y, z)):
            lo, hi = min(self.p1[q], self.p2[q]), max(self.p1[q], self.p2[q])
            r = r & (v >= lo - tol) & (v <= hi + tol)
        return r


def _transform_matrix(el) -> np.ndarray:
    """The 4×4 matrix of a CSXCAD <Transformation>: its operations applied
    to the primitive in the order written (Translate, Rotate_X/Y/Z by an
    angle in radians, Rotate_Origin about an axis through the origin, Scale,
    Scale3, Matrix given row by row)."""
    M = np.eye(4)
    for op in el:
        a = [float(v) for v in op.get("Argument", "").split(",") if v.strip()]
        T = np.eye(4)
        if op.tag == "Translate":
            T[:3, 3] = a[:3]
        elif op.tag in ("Rotate_X", "Rotate_Y", "Rotate_Z", "Rotate_Origin"):
            if op.tag == "Rotate_Origin":
                ax, ang = np.array(a[:3]), a[3]
            else:
                ax, ang = np.eye(3)["XYZ".index(op.tag[-1])], a[0]
            k = ax / np.linalg.norm(ax)
            K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
            T[:3, :3] = np.eye(3) + math.sin(ang) * K + (1.0 - math.cos(ang)) * (K @ K)
        elif op.tag == "Scale":
            T[:3, :3] *= a[0]
        elif op.tag == "Scale3":
            T[:3, :3] = np.diag(a[:3])
        elif op.tag == "Matrix":
            T = np.array(a[:16]).reshape(4, 4)
        else:
            raise NotImplementedError(f"transformation {op.tag}")
        M = T @ M
    return M


@dataclass
class Transformed:
    """A primitive under a transformation: the inside test of the
    primitive at the point mapped back, with the tolerance divided by the
    transformation's smallest singular value (src/compile/openems.rs:
    12-16); ``p1``/``p2`` the transformed bounding box."""
    prim: object
    M: np.ndarray
    priority: int
    p1: tuple = ()
    p2: tuple = ()

    def __post_init__(self):
        self.Minv = np.linalg.inv(self.M)
        self.smin = float(np.linalg.svd(self.M[:3, :3], compute_uv=False).min())
        c = np.array([[x, y, z, 1.0] for x in (self.prim.p1[0], self.prim.p2[0])
                      for y in (self.prim.p1[1], self.prim.p2[1]) for z in (self.prim.p1[2], self.prim.p2[2])])
        w = (self.M @ c.T)[:3]
        self.p1, self.p2 = tuple(w.min(axis=1)), tuple(w.max(axis=1))

    def inside(self, x, y, z, tol):
        R = self.Minv
        loc = [R[r, 0] * x + R[r, 1] * y + R[r, 2] * z + R[r, 3] for r in range(3)]
        return self.prim.inside(loc[0], loc[1], loc[2], tol / self.smin)


@dataclass
class LinPoly:
    """An extruded polygon (CSXCAD LinPoly): vertices (X1, X2) in the plane
    normal to ``normal`` (X1 along the next axis, X2 along the one after),
    from ``elevation`` over ``length``; the inside test closed, the polygon
    grown by the tolerance along the bisectors of its corners and the
    extrusion by the tolerance at both ends (src/compile/openems.rs:
    386-460)."""
    normal: int
    elevation: float
    length: float
    vertices: list
    priority: int
    p1: tuple = ()
    p2: tuple = ()

    def __post_init__(self):
        n, u, w = self.normal, (self.normal + 1) % 3, (self.normal + 2) % 3
        lo, hi = [0.0] * 3, [0.0] * 3
        lo[n], hi[n] = sorted((self.elevation, self.elevation + self.length))
        lo[u], hi[u] = min(v[0] for v in self.vertices), max(v[0] for v in self.vertices)
        lo[w], hi[w] = min(v[1] for v in self.vertices), max(v[1] for v in self.vertices)
        self.p1, self.p2 = tuple(lo), tuple(hi)

    def _grown(self, t):
        v = self.vertices
        k = len(v)
        area = sum(v[i][0] * v[(i + 1) % k][1] - v[(i + 1) % k][0] * v[i][1] for i in range(k))
        sign = 1.0 if area >= 0.0 else -1.0

        def normal(i):
            a, b = v[i], v[(i + 1) % k]
            dx, dy = b[0] - a[0], b[1] - a[1]
            ln = math.hypot(dx, dy)
            return (sign * dy / ln, -sign * dx / ln) if ln > 0 else None

        out = []
        for i in range(k):
            prev = next((normal((i - j) % k) for j in range(1, k) if normal((i - j) % k)), None)
            q = normal(i)
            if prev and q:
                d = 1.0 + prev[0] * q[0] + prev[1] * q[1]
                m = ((prev[0] + q[0]) / d, (prev[1] + q[1]) / d) if d > 1e-6 else q
            else:
                m = prev or q or (0.0, 0.0)
            out.append((v[i][0] + t * m[0], v[i][1] + t * m[1]))
        return out

    def inside(self, x, y, z, tol):
        c = [np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64), np.asarray(z, dtype=np.float64)]
        n, u, w = self.normal, (self.normal + 1) % 3, (self.normal + 2) % 3
        lo, hi = sorted((self.elevation, self.elevation + self.length))
        r = (c[n] >= lo - tol) & (c[n] <= hi + tol)
        P, Q = np.broadcast_arrays(c[u], c[w])
        g = self._grown(tol)
        ins = np.zeros(P.shape, dtype=bool)
        for i in range(len(g)):
            (x0, y0), (x1, y1) = g[i], g[(i + 1) % len(g)]
            cross = ((y0 > Q) != (y1 > Q))
            with np.errstate(all="ignore"):
                xi = x0 + (Q - y0) * (x1 - x0) / (y1 - y0)
            ins ^= cross & (P < xi)
        return r & ins


@dataclass
class Polyhedron:
    """A closed triangle mesh (CSXCAD Polyhedron): vertices and faces
    (vertex index triples); inside where the solid angle its faces subtend
    sums to 4π, or 2π on a face (the generalised winding number, van
    Oosterom and Strackee's triangle solid angle; closed), not grown by the
    inside tolerance (the
    reference grows only the primitives it lists, src/compile/openems.rs:
    459-525); ``p1``/``p2`` its bounding box."""
    vertices: list
    faces: list
    priority: int
    p1: tuple = ()
    p2: tuple = ()

    def __post_init__(self):
        self.p1 = tuple(min(v[a] for v in self.vertices) for a in range(3))
        self.p2 = tuple(max(v[a] for v in self.vertices) for a in range(3))

    def inside(self, x, y, z, tol):
        c = np.broadcast_arrays(np.asarray(x, np.float64), np.asarray(y, np.float64), np.asarray(z, np.float64))
        total = np.zeros(c[0].shape)
        for f in self.faces:
            r = [[self.vertices[i][q] - c[q] for q in range(3)] for i in f]
            (ax, ay, az), (bx, by, bz), (cx, cy, cz) = r
            det = ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx)
            la = np.sqrt(ax * ax + ay * ay + az * az)
            lb = np.sqrt(bx * bx + by * by + bz * bz)
            lc = np.sqrt(cx * cx + cy * cy + cz * cz)
            den = (la * lb * lc + (ax * bx + ay * by + az * bz) * lc + (ax * cx + ay * cy + az * cz) * lb
                   + (bx * cx + by * cy + bz * cz) * la)
            total += 2.0 * np.arctan2(det, den)
        # 4π inside, 0 outside, 2π on a face: closed, as CSXCAD's inside tests.
        return np.abs(total) > math.pi


@dataclass
class Wire:
    """A wire (CSXCAD Wire): the points within ``radius`` of its polyline
    (segments with round ends), closed; grown by the inside tolerance
    (src/compile/openems.rs:509-512); ``p1``/``p2`` its bounding box."""
    points: list
    radius: float
    priority: int
    p1: tuple = ()
    p2: tuple = ()

    def __post_init__(self):
        self.p1 = tuple(min(p[a] for p in self.points) - self.radius for a in range(3))
        self.p2 = tuple(max(p[a] for p in self.points) + self.radius for a in range(3))

    def inside(self, x, y, z, tol):
        c = np.broadcast_arrays(np.asarray(x, np.float64), np.asarray(y, np.float64), np.asarray(z, np.float64))
        r2 = (self.radius + tol) ** 2
        out = np.zeros(c[0].shape, dtype=bool)
        pts = self.points if len(self.points) > 1 else self.points * 2
        for a, b in zip(pts[:-1], pts[1:]):
            d = [b[q] - a[q] for q in range(3)]
            dd = sum(v * v for v in d)
            t = sum((c[q] - a[q]) * d[q] for q in range(3)) / dd if dd > 0 else np.zeros(c[0].shape)
            t = np.clip(t, 0.0, 1.0)
            dist2 = sum((c[q] - (a[q] + t * d[q])) ** 2 for q in range(3))
            out |= dist2 <= r2
        return out


@dataclass
class Shape:
    """A sphere, spherical shell, cylinder or cylindrical shell primitive
    (CSXCAD's closed inside tests, grown by openEMS's inside tolerance;
    src/compile/openems.rs:5-35); ``p1``/``p2`` its bounding box."""
    kind: str
    a: tuple             # centre (spheres) or first axis point (cylinders)
    b: tuple             # second axis point (cylinders)
    radius: float
    width: float         # shell width (0: solid)
    priority: int
    p1: tuple = ()
    p2: tuple = ()

    def __post_init__(self):
        r = self.radius + 0.5 * self.width
        pts = [self.a] if self.kind in ("Sphere", "SphericalShell") else [self.a, self.b]
        self.p1 = tuple(min(p[q] for p in pts) - r for q in range(3))
        self.p2 = tuple(max(p[q] for p in pts) + r for q in range(3))

    def inside(self, x, y, z, tol):
        d = [np.asarray(v, dtype=np.float64) - self.a[q] for q, v in enumerate((x, y, z))]
        if self.kind in ("Sphere", "SphericalShell"):
            rad = np.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2)
            along = None
        else:
            ax = np.array(self.b, dtype=np.float64) - np.array(self.a, dtype=np.float64)
            length = float(np.sqrt(np.sum(ax * ax)))
            u = ax / length
            along = d[0] * u[0] + d[1] * u[1] + d[2] * u[2]
            rad = np.sqrt(np.maximum(d[0] ** 2 + d[1] ** 2 + d[2] ** 2 - along ** 2, 0.0))
        if self.width > 0.0:
            r = np.abs(rad - self.radius) <= 0.5 * self.width + tol
        else:
            r = rad <= self.radius + tol
        if along is not None:
            r = r & (along >= -tol) & (along <= length + tol)
        return r


@dataclass
class Prop:
    kind: str            # Material, Metal, Excitation, ProbeBox
    name: str
    attrs: dict
    prop: dict = field(default_factory=dict)
    boxes: list = field(default_factory=list)
    fd: list = field(default_factory=list)
    order: int = 0
    # Weighting functions of a material's Epsilon, Mue, Kappa, Sigma: per
    # quantity three expressions in x, y, z (drawing units), None for 1.
    weight: dict = field(default_factory=dict)
    # The property's user attributes (its <Attributes> child: a waveguide
    # probe's ModeFunctionX/Y/Z).
    user: dict = field(default_factory=dict)


@dataclass
class OpenEmsFile:
    lines: list          # drawing units, per axis
    unit: float
    max_steps: int
    end_criteria: float
    max_time: float | None
    timestep: float | None
    timestep_factor: float
    timestep_method: int
    oversampling: int
    signal: Signal
    faces: list          # per face (kind, parameter)
    mur_velocity: float | None
    props: list
    background: dict | None = None
    cell_constant: bool = False   # CellConstantMaterial: cell-centre materials
    f_max: float | None = None    # <FDTD f_max>: the explicit highest frequency
    notes: list = field(default_factory=list)  # warnings of the reading
    dumps: list = field(default_factory=list)  # (name, DumpType) of the file's DumpBoxes


def _f(x, default=None):
    return default if x is None else float(x)


def _vec3(text, default, isotropic=True):
    """A material value: isotropic materials take the first number for all
    three axes; anisotropic ones (Isotropy="0") take the numbers given for
    x, y, z in turn, the missing ones the default."""
    if text is None:
        return [default] * 3
    v = [float(x) for x in text.split(",")]
    if isotropic:
        return [v[0]] * 3
    return (v + [default] * 3)[:3]


def _face(v: str):
    """openEMS's reading of a boundary name (src/io/openems/model.rs:11-18):
    PEC, PMC, MUR and PML_<n> case sensitive; a value starting with a digit
    or sign by its integer prefix (0 PEC, 1 PMC, 2 MUR, 3 PML_8, else PEC);
    PML_<n> by the integer prefix of <n> (n <= 0: PEC); anything else PEC."""
    if v and (v[0].isdigit() or v[0] in "+-"):
        m = re.match(r"[+-]?\d+", v)
        k = int(m.group(0)) if m else 0
        return {1: (PMC_FACE, None), 2: (MUR_FACE, None), 3: (PML_FACE, 8)}.get(k, (PEC_FACE, None))
    if v == "PMC":
        return (PMC_FACE, None)
    if v == "MUR":
        return (MUR_FACE, None)
    if v.startswith("PML_"):
        m = re.match(r"[+-]?\d+", v[4:])
        if m and int(m.group(0)) > 0:
            return (PML_FACE, int(m.group(0)))
    return (PEC_FACE, None)


def _parameters(root):
    """The file's <ParameterSet> constants substituted into the numeric
    attributes of primitives and material properties (openEMS evaluates
    them there); the document re-parsed if any were given."""
    ps = root.find("ContinuousStructure/ParameterSet")
    if ps is None:
        return root
    env = {}
    for p in ps:
        if p.get("name") is not None and p.get("value") is not None:
            env[p.get("name")] = float(p.get("value"))
    if not env:
        return root

    def number(t):
        try:
            float(t)
            return t
        except ValueError:
            return repr(float(Expression(t, tuple(env)).evaluate(**env)))

    pr = root.find("ContinuousStructure/Properties")
    for el in (pr.iter() if pr is not None else []):
        if el.tag in ("Weight", "Attributes"):
            continue
        for k, v in list(el.attrib.items()):
            if k in ("Name", "Function"):
                continue
            parts = v.split(",")
            try:
                el.set(k, ",".join(number(x.strip()) for x in parts))
            except ValueError:
                pass
    return root


def read_stl(path: str) -> list:
    """The triangles of an STL file, ASCII or binary: [(v0, v1, v2)]."""
    with open(path, "rb") as h:
        data = h.read()
    if data[:5].lower() == b"solid" and b"facet" in data[:1024]:
        verts = [tuple(float(x) for x in ln.split()[1:4]) for ln in data.decode("ascii", "replace").splitlines()
                 if ln.strip().startswith("vertex")]
        if len(verts) % 3:
            raise ValueError(f"{path}: vertices not in threes")
        return [tuple(verts[3 * i:3 * i + 3]) for i in range(len(verts) // 3)]
    n = struct.unpack_from("<I", data, 80)[0]
    if len(data) < 84 + 50 * n:
        raise ValueError(f"{path}: truncated binary STL")
    tris = []
    for i in range(n):
        v = struct.unpack_from("<12f", data, 84 + 50 * i)
        tris.append(((v[3], v[4], v[5]), (v[6], v[7], v[8]), (v[9], v[10], v[11])))
    return tris


def parse(text: str, base_dir: str | None = None) -> OpenEmsFile:
    """An openEMS model file; ``base_dir``: where files it names (STL
    meshes) are read from (the current directory without one)."""
    root = _parameters(ET.fromstring(text))
    fd = root.find("FDTD")
    if fd is None:
        raise ValueError("no <FDTD> element")
    ex = fd.find("Excitation")
    if ex is None:
        raise ValueError("no excitation signal")
    kind = int(float(ex.get("Type", "0")))
    if kind == 0:
        sig = Signal(0, float(ex.get("f0")), float(ex.get("fc")))
    elif kind == 1:
        sig = Signal(1, float(ex.get("f0")))
    elif kind in (2, 3):
        sig = Signal(kind)
    elif kind == 10:
        sig = Signal(10, _f(ex.get("f0"), 0.0), expr=Expression(ex.get("Function")))
    else:
        raise NotImplementedError(f"excitation signal type {kind}")
    bc = fd.find("BoundaryCond")
    faces = []
    for name in FACE_NAMES:
        faces.append(_face((bc.get(name) if bc is not None else None) or "PEC"))
    mur_v = _f(bc.get("MUR_PhaseVelocity")) if bc is not None else None
    cs = root.find("ContinuousStructure")
    grid = cs.find("RectilinearGrid")
    if int(float(grid.get("CoordSystem", cs.get("CoordSystem", "0")))) != 0:
        raise NotImplementedError("cylindrical grids")
    unit = float(grid.get("DeltaUnit", "1"))
    lines = []
    for tag in ("XLines", "YLines", "ZLines"):
        v = sorted(set(float(x) for x in grid.find(tag).text.split(",")))  # openEMS sorts, drops repeats
        lines.append(v)
    props = []
    notes: list[str] = []
    pr = cs.find("Properties")
    dumps: list[tuple[str, int]] = []
    for q, el in enumerate(list(pr) if pr is not None else []):
        if el.tag == "DumpBox":
            # A field dump only writes files: the fields, the steps and
            # every probe are the same with or without it. Its files are in
            # openEMS's HDF5/VTK layout (src/io/openems/dump.rs), which this
            # reader does not write; the run's probe files are.
            dumps.append((el.get("Name", ""), int(float(el.get("DumpType", "0")))))
            notes.append(f"dump {el.get('Name', '')!r}: openEMS's dump files are not written")
            continue
        boxes = []
        only_long_cylinders = False  # a probe whose primitives openEMS writes nothing for
        prims = el.find("Primitives")
        def pt(e):
            return tuple(float(e.get(c)) for c in "XYZ")

        for b in (list(prims) if prims is not None else []):
            if el.tag == "LumpedElement" and b.tag != "Box":
                # src/io/openems/model.rs:396-411: openEMS places lumped
                # elements on boxes only and skips other primitives.
                notes.append(f"lumped element {el.get('Name', '')!r}: a {b.tag} primitive is not supported by "
                             "openEMS (boxes only); skipped, as openEMS does")
                continue
            tr = b.find("Transformation")
            if tr is not None and (el.tag not in MATERIALS + ("Metal",) or b.tag not in
                                   ("Box", "Sphere", "SphericalShell", "Cylinder", "CylindricalShell")):
                raise NotImplementedError("transformed primitives")
            if b.get("CoordSystem", "0") != "0":
                raise NotImplementedError(f"primitive {b.tag} in cylindrical coordinates")
            prio = int(float(b.get("Priority", "0")))
            if b.tag == "Box":
                boxes.append(Box(pt(b.find("P1")), pt(b.find("P2")), prio))
            elif b.tag == "MultiBox":
                starts, ends = b.findall("StartP"), b.findall("EndP")
                boxes += [Box(pt(s0), pt(e0), prio) for s0, e0 in zip(starts, ends)]
            elif b.tag in ("Cylinder", "CylindricalShell") and el.tag == "ProbeBox" and tr is None:
                # A probe on a zero-length cylinder is a point probe; openEMS
                # writes no file for one on a longer cylinder.
                if pt(b.find("P1")) == pt(b.find("P2")):
                    boxes.append(Box(pt(b.find("P1")), pt(b.find("P2")), prio))
                else:
                    only_long_cylinders = True
            elif b.tag == "LinPoly" and el.tag in MATERIALS + ("Metal",) and tr is None:
                verts = [(float(q.get("X1")), float(q.get("X2"))) for q in b.findall("Vertex")]
                boxes.append(LinPoly(int(float(b.get("NormDir", "2"))), float(b.get("Elevation", "0")),
                                     float(b.get("Length", "0")), verts, prio))
            elif b.tag == "Polyhedron" and el.tag in MATERIALS + ("Metal",) and tr is None:
                verts = [tuple(float(x) for x in v.text.split(",")) for v in b.findall("Vertex")]
                tri = [tuple(int(x) for x in f_.text.split(",")) for f_ in b.findall("Face")]
                if not verts or not tri or any(len(f_) != 3 or max(f_) >= len(verts) for f_ in tri):
                    raise NotImplementedError(f"polyhedron in {el.get('Name')!r}: faces other than triangles")
                boxes.append(Polyhedron(verts, tri, prio))
            elif b.tag == "PolyhedronReader" and el.tag in MATERIALS + ("Metal",) and tr is None:
                if b.get("FileType", "STL").upper() != "STL":
                    raise NotImplementedError(f"PolyhedronReader in {el.get('Name')!r}: file type "
                                              f"{b.get('FileType')!r}")
                tris = read_stl(os.path.join(base_dir or ".", b.get("FileName", "")))
                verts = [v for t in tris for v in t]
                boxes.append(Polyhedron(verts, [(3 * i, 3 * i + 1, 3 * i + 2) for i in range(len(tris))], prio))
            elif b.tag == "Wire" and el.tag == "Metal" and tr is None:
                radius = float(b.get("WireRadius", "0"))
                if radius < 0.5 * min(float(np.min(np.diff(v))) for v in lines if len(v) > 1):
                    # Thinner wires get an in-cell correction (the reference's
                    # compile::wire), not restated.
                    raise NotImplementedError(f"wire {el.get('Name')!r} thinner than half the smallest cell")
                boxes.append(Wire([pt(v) for v in b.findall("Vertex")], radius, prio))
            elif b.tag == "Polygon" and el.tag in ("Metal", "ConductingSheet") and tr is None:
                # A flat polygon: an extruded one of length 0.
                verts = [(float(q.get("X1")), float(q.get("X2"))) for q in b.findall("Vertex")]
                boxes.append(LinPoly(int(float(b.get("NormDir", "2"))), float(b.get("Elevation", "0")), 0.0,
                                     verts, prio))
            elif b.tag in ("Sphere", "SphericalShell", "Cylinder", "CylindricalShell") and \
                    el.tag in MATERIALS + ("Metal", "Excitation"):
                sph = b.tag.startswith("Spher")
                a0 = pt(b.find("Center")) if sph else pt(b.find("P1"))
                b0 = a0 if sph else pt(b.find("P2"))
                boxes.append(Shape(b.tag, a0, b0, float(b.get("Radius")),
                                   float(b.get("ShellWidth", "0")) if b.tag.endswith("Shell") else 0.0, prio))
            else:
                raise NotImplementedError(f"primitive {b.tag} in {el.get('Name')!r}")
            if tr is not None:
                boxes[-1] = Transformed(boxes[-1], _transform_matrix(tr), prio)
        if el.tag not in ("Material", "Metal", "Excitation", "ProbeBox", "LorentzMaterial", "DebyeMaterial",
                          "LumpedElement", "ConductingSheet", "AbsorbingBC"):
            raise NotImplementedError(f"property {el.tag}")
        if el.tag == "ProbeBox" and not boxes and only_long_cylinders:
            continue
        if el.tag == "ProbeBox" and any(not isinstance(b, Box) for b in boxes):
            raise NotImplementedError(f"probe {el.get('Name')!r} on a primitive other than a box")
        weight = {}
        wel = el.find("Weight")
        if wel is not None and el.tag == "Excitation":
            if set(wel.attrib) - {"X", "Y", "Z"}:
                raise NotImplementedError(f"weighting functions ({el.get('Name')!r})")
            weight["Excite"] = [None if wel.get(c, "1").strip() in ("1", "1.0") else
                                Expression(wel.get(c), ("x", "y", "z")) for c in "XYZ"]
        elif wel is not None:
            poles = {"EpsilonPlasmaFrequency", "EpsilonLorPoleFrequency", "EpsilonRelaxTime", "EpsilonDelta",
                     "MuePlasmaFrequency", "MueLorPoleFrequency", "MueRelaxTime", "MueDelta"}
            allowed = {"Epsilon", "Mue", "Kappa", "Sigma"} | (poles if el.tag != "Material" else set())
            if el.tag not in MATERIALS or set(wel.attrib) - allowed:
                raise NotImplementedError(f"weighting functions ({el.get('Name')!r})")
            iso = el.get("Isotropy", "1") != "0"
            for key, text in wel.attrib.items():
                parts = [t.strip() for t in text.split(",")]
                parts = [parts[0]] * 3 if iso else (parts + ["1"] * 3)[:3]
                weight[key] = [None if t in ("1", "1.0") else Expression(t, ("x", "y", "z")) for t in parts]
        sub = el.find("Property")
        fds = el.find("FD_Samples")
        fd_list = [float(x) for x in fds.text.split(",")] if fds is not None and fds.text else []
        if el.tag == "ProbeBox" and len(boxes) > 1:
            # Several primitives: several probes <name>_0, <name>_1, … in
            # primitive order, one file each (src/io/openems/model.rs:27-29).
            for t, b in enumerate(boxes):
                props.append(Prop(el.tag, f"{el.get('Name', '')}_{t}", dict(el.attrib),
                                  dict(sub.attrib) if sub is not None else {}, [b], fd_list, q, weight))
            continue
        user_el = el.find("Attributes")
        props.append(Prop(el.tag, el.get("Name", ""), dict(el.attrib), dict(sub.attrib) if sub is not None else {},
                          boxes, fd_list, q, weight, dict(user_el.attrib) if user_el is not None else {}))
    # src/fdtd/convert.rs:32-47: OverSampling below 2 → 4; endCriteria
    # absent or 0 → openEMS's default, negative → none; TimeStepFactor
    # outside (0, 1] → 1 and TimeStepMethod other than 1 or 3 → 1 (what
    # openEMS does).
    os_ = int(float(fd.get("OverSampling", "4")))
    end = float(fd.get("endCriteria", "0"))
    end = 1e-6 if end == 0.0 else (None if end < 0 else end)  # openEMS default: -60 dB
    factor = float(fd.get("TimeStepFactor", "1"))
    method = int(float(fd.get("TimeStepMethod", "3")))
    bg = cs.find("BackgroundMaterial")
    for el in cs:
        if el.tag not in ("Properties", "RectilinearGrid", "BackgroundMaterial", "ParameterSet"):
            raise NotImplementedError(f"<{el.tag}> in the structure")
    return OpenEmsFile(lines, unit, int(float(fd.get("NumberOfTimesteps", "0"))), end,
                       _f(fd.get("MaxTime")), _f(fd.get("TimeStep")),
                       factor if 0.0 < factor <= 1.0 else 1.0, method if method in (1, 3) else 1,
                       os_ if os_ >= 2 else 4, sig, faces, mur_v, props,
                       dict(bg.attrib) if bg is not None else None,
                       fd.get("CellConstantMaterial", "0") not in ("0", "false", "False"), _f(fd.get("f_max")),
                       notes, dumps)


# ---------------------------------------------------------------------------
# Snapping (src/sim/map.rs:1816-1870).

def _box_nodes(lo, hi):
    """The nodes of the inclusive box lo..hi."""
    return [(i, j, k) for i in range(lo[0], hi[0] + 1) for j in range(lo[1], hi[1] + 1)
            for k in range(lo[2], hi[2] + 1)]


def snap_lower(lines, x):
    best = 0
    for i in range(1, len(lines)):
        tol = 1e-9 * abs(lines[i] - lines[i - 1])
        if abs(lines[i] - x) < abs(lines[best] - x) - tol:
            best = i
    return best


def snap_upper(lines, x):
    best = 0
    for i in range(1, len(lines)):
        tol = 1e-9 * abs(lines[i] - lines[i - 1])
        if abs(lines[i] - x) <= abs(lines[best] - x) + tol:
            best = i
    return best


def snap_cell(lines, x):
    if len(lines) < 2:
        return 0
    i = 0
    for k in range(1, len(lines) - 1):
        tol = 1e-9 * abs(lines[k + 1] - lines[k - 1])
        if lines[k] < x - tol:
            i = k
    return i


def voltage_path(start, stop):
    """src/sim/map.rs:1683-1702: x, then y, then z; reversed edges −1."""
    out, p = [], list(start)
    for a in range(3):
        lo, hi = p[a], stop[a]
        if lo <= hi:
            for i in range(lo, hi):
                p[a] = i
                out.append((a, tuple(p), 1.0))
        else:
            for i in range(lo - 1, hi - 1, -1):
                p[a] = i
                out.append((a, tuple(p), -1.0))
        p[a] = hi
    return out


def loop_entries(n, lo, hi, layer):
    """−∮H around the E edges along n with transverse nodes in lo..hi
    (src/engine/port.rs:231-260)."""
    b, c = (n + 1) % 3, (n + 2) % 3

    def node(pb, pc):
        p = [0, 0, 0]
        p[n], p[b], p[c] = layer, pb, pc
        return tuple(p)

    v = []
    for pc in range(lo[c], hi[c] + 1):
        v.append((c, node(hi[b], pc), -1.0))
        if lo[b] > 0:
            v.append((c, node(lo[b] - 1, pc), 1.0))
    for pb in range(lo[b], hi[b] + 1):
        v.append((b, node(pb, hi[c]), 1.0))
        if lo[c] > 0:
            v.append((b, node(pb, lo[c] - 1), -1.0))
    return v


def openems_loop_order(entries, n, lo, hi):
    """src/sim/map.rs:1776-1805."""
    b, c = (n + 1) % 3, (n + 2) % 3

    def key(e):
        a, p, _ = e
        if a == b and p[c] < lo[c]:
            return (0, p[b])
        if a == c and p[b] >= hi[b]:
            return (1, p[c])
        if a == b:
            return (2, p[b])
        return (3, p[c])

    return sorted(entries, key=key)


# ---------------------------------------------------------------------------
# Set-up.

@dataclass
class ProbeSpec:
    name: str
    kind: str            # voltage, current, efield, hfield
    ops: list            # engine op indices (one, or three for field probes)
    location: tuple
    fd: list
    oversampling: int | None = None
    start_time: float = 0.0
    stop_time: float = 0.0
    # Waveguide probes: (weight, [(area, mode (2,), (op x, op y))]) for the
    # mode purity column.
    purity: tuple | None = None


class Setup:
    """A parsed file mapped onto a built ``ems_b200.Model``: ``model``,
    ``dt``, ``steps`` (the run length), ``probes`` and ``warnings``."""

    def __init__(self, f: OpenEmsFile):
        from . import PEC, PMC, Model
        self.file = f
        self.warnings: list[str] = list(f.notes)
        u = f.unit
        lines_m = [np.array(v) * u for v in f.lines]
        n = [len(v) for v in f.lines]
        self.nodes = n
        m = Model(*lines_m)
        self.lines_m = lines_m
        m.faces([PMC if k == PMC_FACE else PEC for k, _ in f.faces])
        # openEMS's inside tolerance of metal, material and excitation
        # primitives: 1e-3 of the smallest cell width, drawing units.
        self.tol = 1e-3 * min(float(np.min(np.diff(v))) for v in f.lines if len(v) > 1)
        self.lumped_edges = {(a, *e) for a, edges in self._lumped_boxes() for e in edges}
        self.sheet_edges: set = set()     # (axis, i, j, k) of the conducting-sheet edges with a circuit
        self.sheet_branches: list = []    # (axis, node, [(L, R), (L, R)])
        self._materials(m)
        if f.cell_constant and any(p.weight or any(not isinstance(b, Box) for b in p.boxes) for p in f.props):
            raise NotImplementedError("weighting functions or round primitives with CellConstantMaterial")
        if not f.cell_constant:
            self._sampled_materials(m)
        # Time step: openEMS's criterion, TimeStepFactor, or TimeStep.
        if f.timestep is not None:
            base = f.timestep
        else:
            base = m.openems_timestep(f.timestep_method)
        dt = f.timestep_factor * base
        if f.signal.kind == 1 and f.signal.f0 > 0:
            period = 1.0 / f.signal.f0
            dt = period / (math.floor(period / dt) + 1.0)
        m.build_bound(dt, openems_rounding=True, openems_sigma_m=True)
        self.dt = dt
        self._sheets(m)
        # Lumped elements with an inductor or in series (openEMS keeps the H
        # edge of their direction and node at a PMC wall, and their E edges).
        self.branch_edges = set()
        for (a, edges), p in zip(self._lumped_boxes(), [q for q in f.props if q.kind == "LumpedElement"]):
            if p.attrs.get("L") is not None or p.attrs.get("LEtype", "0") not in ("0", "-1"):
                self.branch_edges |= {(a, *e) for e in edges}
        self._pmc_half_cell(m)
        self.upml_op = None
        if any(k == PML_FACE for k, _ in f.faces):
            self.upml_op = m.add_openems_pml([c if k == PML_FACE else 0 for k, c in f.faces])
            self.upml_h = m.upml_table(self.upml_op)[1]
        self._lumped(m)
        # openEMS's Mur faces take the interior neighbours before the
        # dispersive correction of their update: the Mur operator is
        # registered before the poles (src/compile/mod.rs:1258-1263).
        self.excited = self._excitation_edges()
        self._mur(m)
        self._dispersive(m)
        self._refuse_poles_beside_mur(m)
        steps = f.max_steps
        if f.max_time is not None and f.max_time > 0:
            steps = min(steps, int(math.floor(f.max_time / dt)))
        self.steps = steps
        self.criterion = f.end_criteria
        self.model = m
        self.h_sources = []
        self._absorbing_sheets(m)
        self._excitations(m)
        self.probes: list[ProbeSpec] = []
        self._probes(m)

    # -- geometry helpers (drawing units)
    def _inside(self, a, x, lo, hi):
        tol = 1e-9 * max(1.0, abs(hi - lo), abs(self.file.lines[a][-1] - self.file.lines[a][0]))
        return lo - tol <= x <= hi + tol

    def _inside_prim(self, x, lo, hi):
        """Closed inside test of metal, materials and excitations with the
        tolerance ``self.tol`` (src/compile/openems.rs:5-30)."""
        return lo - self.tol <= x <= hi + self.tol

    def _sampled_materials(self, m):
        """Edge materials from point samples the openEMS way (csx's
        sub-cell discretisation with openEMS's rules, src/compile/
        openems.rs:36-60 and 83-98): an E edge along a averages eps_r and
        kappa over the quarters of its dual face, sampled at the edge's
        midpoint along a and a quarter of the adjacent cell widths either
        side in the other axes, area-weighted; an H dual edge along a
        combines mu_r over the two halves of the dual edge, sampled at the
        face centre across and at x_n -+ dx/4 along a, length-weighted
        harmonic, and sigma_m by openEMS's rule (harmonic, a lossless upper
        half gives 0, a lossless lower half is left out). Each sample takes
        the highest-priority material containing it (closed, with the
        inside tolerance; at equal priority the one defined first), metal
        not counted, else the background. Faces of the domain see their
        in-domain parts only."""
        f = self.file
        n = self.nodes
        lines = [np.asarray(v, dtype=np.float64) for v in f.lines]
        d = [np.diff(v) for v in lines]
        bg = f.background
        props = []
        items = []
        weights = {}  # property index in the table -> weighting functions
        for p in f.props:
            if p.kind not in MATERIALS:
                continue
            iso = p.attrs.get("Isotropy", "1") != "0"
            props.append([_vec3(p.prop.get(k), dv, iso) for k, dv in
                          (("Epsilon", 1.0), ("Kappa", 0.0), ("Mue", 1.0), ("Sigma", 0.0))])
            if p.weight:
                weights[len(props)] = p.weight
            for b in p.boxes:
                items.append((b.priority, -p.order, len(props) - 1, b))
        items.sort(key=lambda t: (t[0], t[1]))
        base = ([_vec3(bg.get(k), dv, True) for k, dv in
                 (("Epsilon", 1.0), ("Kappa", 0.0), ("Mue", 1.0), ("Sigma", 0.0))]
                if bg else [[1.0] * 3, [0.0] * 3, [1.0] * 3, [0.0] * 3])
        table = np.array([base] + props, dtype=np.float64)  # [prop, quantity, axis]
        qname = ("Epsilon", "Kappa", "Mue", "Sigma")

        def value(pid, q, a, xs):
            """Quantity q along a of the samples' materials, each weighted
            at its sample point (the weighting function of the winning
            material times its value)."""
            v = table[pid, q, a]
            for idx, wt in weights.items():
                w = wt.get(qname[q])
                if not w or w[a] is None:
                    continue
                I = np.nonzero(pid == idx)
                if I[0].size:  # (v is a copy: pid indexes the table)
                    v[I] = v[I] * w[a].evaluate(x=xs[0][I[0]], y=xs[1][I[1]], z=xs[2][I[2]])
            return v

        def winner(xs):
            """Property index (0 background) on the grid of coordinates xs."""
            idx = np.zeros([len(x) for x in xs], dtype=np.int64)
            for _, _, pi, b in items:
                mask = np.broadcast_to(b.inside(xs[0][:, None, None], xs[1][None, :, None], xs[2][None, None, :],
                                                self.tol), idx.shape)
                idx[mask] = pi + 1
            return idx

        def sides(q):
            """Sample coordinates and weights of the lower and upper halves
            around each node line of axis q (weight 0 outside)."""
            x = lines[q]
            lo_w = np.zeros(n[q])
            hi_w = np.zeros(n[q])
            lo_x = x.copy()
            hi_x = x.copy()
            if n[q] > 1:
                lo_w[1:] = 0.5 * d[q]
                hi_w[:-1] = 0.5 * d[q]
                lo_x[1:] = x[1:] - 0.25 * d[q]
                hi_x[:-1] = x[:-1] + 0.25 * d[q]
            return [(lo_x, lo_w), (hi_x, hi_w)]

        def centres(q):
            x = lines[q]
            c = np.ones(n[q]) * x[-1]
            if n[q] > 1:
                c[:-1] = 0.5 * (x[:-1] + x[1:])
            return c

        for a in range(3):
            b, c = (a + 1) % 3, (a + 2) % 3
            # E edges along a.
            num_e = np.zeros(n)
            num_k = np.zeros(n)
            den = np.zeros(n)
            for xb, wb in sides(b):
                for xc, wc in sides(c):
                    xs = [None] * 3
                    xs[a], xs[b], xs[c] = centres(a), xb, xc
                    w = np.ones(n)
                    shape = [1, 1, 1]
                    shape[b] = n[b]
                    w = w * wb.reshape(shape)
                    shape = [1, 1, 1]
                    shape[c] = n[c]
                    w = w * wc.reshape(shape)
                    pid = winner(xs)
                    num_e += w * value(pid, 0, a, xs)
                    num_k += w * value(pid, 1, a, xs)
                    den += w
            ok = den > 0
            eps = np.where(ok, num_e / np.where(ok, den, 1.0), 1.0)
            kap = np.where(ok, num_k / np.where(ok, den, 1.0), 0.0)
            m.set_edge_materials(0, a, eps, kap)
            # H dual edges along a.
            length = np.zeros(n)
            inv_mu = np.zeros(n)
            inv_sg = np.zeros(n)
            hi_zero = np.zeros(n, dtype=bool)
            for side, (xa, wa) in enumerate(sides(a)):
                xs = [None] * 3
                xs[a], xs[b], xs[c] = xa, centres(b), centres(c)
                shape = [1, 1, 1]
                shape[a] = n[a]
                w = np.broadcast_to(wa.reshape(shape), n)
                pid = winner(xs)
                mu = value(pid, 2, a, xs)
                sg = value(pid, 3, a, xs)
                has = w > 0
                length += w
                inv_mu += np.where(has, w / mu, 0.0)
                inv_sg += np.where(has & (sg != 0.0), w / np.where(sg != 0.0, sg, 1.0), 0.0)
                if side == 1:
                    hi_zero |= has & (sg == 0.0)
            ok = length > 0
            mu_e = np.where(ok, length / np.where(ok, inv_mu, 1.0), 1.0)
            sg_e = np.where(ok & ~hi_zero & (inv_sg > 0), length / np.where(inv_sg > 0, inv_sg, 1.0), 0.0)
            m.set_edge_materials(1, a, mu_e, sg_e)

    def _materials(self, m):
        f = self.file
        mats = [p for p in f.props if p.kind in ("Metal",) + MATERIALS]
        # Paint in priority order; at equal priority the property defined
        # first wins (it is painted last).
        items = []
        for p in mats:
            for b in p.boxes:
                items.append((b.priority, -p.order, p, b))
        items.sort(key=lambda t: (t[0], t[1]))
        lines = f.lines
        if f.background:
            n = self.nodes
            m.fill(m.cells().box([0, 0, 0], [n[0] - 1, n[1] - 1, n[2] - 1]), self._material(m, f.background))
        cen = [0.5 * (np.array(v[1:]) + np.array(v[:-1])) for v in lines]
        for _, _, p, b in items:
            lo = [min(b.p1[a], b.p2[a]) for a in range(3)]
            hi = [max(b.p1[a], b.p2[a]) for a in range(3)]
            if p.kind == "Metal":
                # Edges whose midpoint lies in the closed primitive, unless
                # a material of higher priority (or of equal priority
                # defined earlier) holds the midpoint too, or the edge is a
                # lumped element's.
                over = [(ob, op) for (_, _, op, ob) in items if op.kind in MATERIALS and
                        (ob.priority > b.priority or (ob.priority == b.priority and op.order < p.order))]
                # A conducting sheet that wins over the metal there makes the
                # edge a sheet edge, not PEC (sheet_over_metal).
                over += [(ob, op) for op in f.props if op.kind == "ConductingSheet" for ob in op.boxes
                         if ob.priority > b.priority or (ob.priority == b.priority and op.order < p.order)]
                n = self.nodes
                for a in range(3):
                    xs = []
                    for q in range(3):
                        v = np.array(lines[q], dtype=np.float64)
                        if q == a:
                            v = np.concatenate([cen[q], [1e30]])  # no edge from the last line
                        shape = [1, 1, 1]
                        shape[q] = n[q]
                        xs.append(v.reshape(shape))
                    mask = np.broadcast_to(b.inside(xs[0], xs[1], xs[2], self.tol), tuple(n)).copy()
                    for ob, _ in over:
                        mask &= ~np.broadcast_to(ob.inside(xs[0], xs[1], xs[2], self.tol), tuple(n))
                    for (a2, i, j, k) in self.lumped_edges:
                        if a2 == a:
                            mask[i, j, k] = False
                    for i, j in zip(*np.nonzero(mask.any(axis=2))):
                        row = np.concatenate([[False], mask[i, j], [False]]).astype(np.int8)
                        st = np.flatnonzero(np.diff(row) == 1)
                        en = np.flatnonzero(np.diff(row) == -1) - 1
                        for k0, k1 in zip(st, en):
                            m.pec_edges(a, [int(i), int(j), int(k0)], [int(i), int(j), int(k1)])
                continue
            if not isinstance(b, Box):
                continue  # round and transformed materials: sampled per edge
            cells = [[i for i, x in enumerate(cen[a]) if self._inside(a, x, lo[a], hi[a])] for a in range(3)]
            if not all(cells):
                continue
            mat = self._material(m, p.prop, p.attrs.get("Isotropy", "1") != "0")
            cs = m.cells().box([c[0] for c in cells], [c[-1] + 1 for c in cells])
            m.fill(cs, mat)

    def _lumped_boxes(self):
        """(axis, edges) of every lumped element: the E edges along its
        direction whose both nodes lie in one of its boxes (closed, the
        boxes snap to the mesh)."""
        out = []
        n, lines = self.nodes, self.file.lines
        for p in self.file.props:
            if p.kind != "LumpedElement":
                continue
            a = int(float(p.attrs.get("Direction", "0")))
            edges = []
            for b in p.boxes:
                lo = [min(b.p1[q], b.p2[q]) for q in range(3)]
                hi = [max(b.p1[q], b.p2[q]) for q in range(3)]
                rng = [[i for i in range(n[q] - (1 if q == a else 0))
                        if self._inside(q, lines[q][i], lo[q], hi[q])
                        and (q != a or self._inside(q, lines[q][i + 1], lo[q], hi[q]))] for q in range(3)]
                edges += [(i, j, k) for i in rng[0] for j in rng[1] for k in rng[2]]
            out.append((a, edges))
        return out

    def _lumped(self, m):
        """Parallel R/C lumped elements the openEMS way (src/sim/map.rs:
        46-255, 540-600, 1525-1680): spread like a homogeneous material
        over their E edges (G_e = g_e·S/R, C_e = g_e·C·S with g_e the edge's
        dual face over its length, outer lines counting full cells, and
        S = Σ over positions along the element of 1/Σ g_e), their R and C
        replacing the medium's conductance and capacitance, and PEC caps
        on the two end planes over the element's whole box (Caps, the
        default). The element's own edges are its own whatever metal lies
        there (they take the medium under the metal,
        src/compile/openems.rs:69-81); on edges inside a PML layer the
        layer replaces the update, so the element's R and C act only
        outside it, spread over all its edges all the same."""
        f = self.file
        n = self.nodes
        boxes = iter(self._lumped_boxes())
        for p in f.props:
            if p.kind != "LumpedElement":
                continue
            a, edges = next(boxes)
            r = _f(p.attrs.get("R"))
            c = _f(p.attrs.get("C"))
            r = r if r is not None and r > 0 and math.isfinite(r) else None
            c = c if c is not None and c > 0 and math.isfinite(c) else None
            ind = _f(p.attrs.get("L"))
            ind = ind if ind is not None and ind > 0 and math.isfinite(ind) else None
            series = p.attrs.get("LEtype", "0") not in ("0", "-1")
            if ind is not None or series:
                self._branch_element(m, p, a, edges, r, ind, c, series)
                continue
            ca, cb = m.coeff(a), m.coeff(3 + a)
            kept, layer = [], []
            for e in edges:
                if cb[e] == 0.0:
                    self.warnings.append(f"lumped element {p.name!r}: edge {e} is PEC (shorted); ignored")
                elif ca[e] == 0.0:  # inside a PML layer: the layer replaces the update
                    layer.append(e)
                else:
                    kept.append(e)
            if layer:
                self.warnings.append(f"lumped element {p.name!r}: {len(layer)} of its {len(kept) + len(layer)} "
                                     "edge(s) lie inside a PML layer and are ignored there")
            if not kept + layer or (r is None and c is None):
                continue

            # openems_edge_geometry (src/sim/map.rs:164-218).
            def geo(e):
                area = 1.0
                for t in range(3):
                    if t == a:
                        continue
                    area *= self.model_dual(t, e[t]) * (2.0 if e[t] in (0, n[t] - 1) else 1.0)
                return area / self.model_delta(a, e[a])

            w = {e: geo(e) for e in kept + layer}
            per = {}
            for e in kept + layer:
                per[e[a]] = per.get(e[a], 0.0) + w[e]
            S = sum(1.0 / x for x in per.values())
            on_sheet = [e for e in kept if (a, *e) in self.sheet_edges]
            if on_sheet:
                self.warnings.append(f"lumped element {p.name!r}: {len(on_sheet)} of its {len(kept) + len(layer)} "
                                     "edge(s) lie on conducting-sheet edges and are ignored there (openEMS's sheet "
                                     "keeps them)")
            for e in kept:
                if (a, *e) in self.sheet_edges:
                    continue
                m.set_edge_circuit(a, e, cap=c * w[e] * S if c is not None else -1.0,
                                   cond=1.0 / (r / (w[e] * S)) if r is not None else -1.0)
            if p.attrs.get("Caps", "1") != "0":
                lo = [min(e[q] for e in kept + layer) for q in range(3)]
                hi = [max(e[q] + (1 if q == a else 0) for e in kept + layer) for q in range(3)]
                for t in range(3):
                    if t == a or hi[t] == lo[t]:
                        continue
                    o = 3 - a - t
                    for plane in (lo[a], hi[a]):
                        blo, bhi = [0, 0, 0], [0, 0, 0]
                        blo[a] = bhi[a] = plane
                        blo[t], bhi[t] = lo[t], hi[t] - 1
                        blo[o], bhi[o] = lo[o], hi[o]
                        if not any((t, *e) in self.sheet_edges for e in _box_nodes(blo, bhi)):
                            m.zero_edges(0, t, blo, bhi)
                            continue
                        for e in _box_nodes(blo, bhi):  # the cap leaves sheet edges alone
                            if (t, *e) not in self.sheet_edges:
                                m.zero_edges(0, t, e, e)

    def _branch_element(self, m, p, a, edges, r, ind, c, series):
        """A lumped element with an inductor or in series the openEMS way
        (src/sim/map.rs:820-1000, 1525-1632; ``Model.add_lumped_openems``):
        caps first, the element's values in csx's equal parts replacing the
        medium of its edges, the edge capacitance limited by the branch
        impedance at the excitation's frequency (series elements; parallel
        ones with an inductor and no capacitor), openEMS's order and, for a
        parallel inductor, its explicit f32 update (the trapezoidal branch
        where that is unstable). An excitation on its edges stays a plain
        soft source, added after the element. Not restated: elements with
        edges in PML layers or on conducting-sheet edges (openEMS installs
        them over the sheet), poles on their edges (openEMS corrects those
        after the element), edge sets that are not one box."""
        n = self.nodes
        if not edges:
            return
        if any((a, *e) in self.sheet_edges for e in edges):
            raise NotImplementedError(f"lumped element {p.name!r}: an inductor or series element on a "
                                      "conducting sheet")
        lo = [min(e[q] for e in edges) for q in range(3)]
        hi = [max(e[q] for e in edges) for q in range(3)]
        box = {(i, j, k) for i in range(lo[0], hi[0] + 1) for j in range(lo[1], hi[1] + 1)
               for k in range(lo[2], hi[2] + 1)}
        box = {e for e in box if e[a] <= hi[a]}
        if set(edges) != box:
            raise NotImplementedError(f"lumped element {p.name!r}: edges that are not one box")
        ca = m.coeff(a)
        if any(ca[e] == 0.0 for e in edges):
            raise NotImplementedError(f"lumped element {p.name!r}: an inductor or series element in a PML layer "
                                      "or on PEC")
        if p.attrs.get("Caps", "1") != "0":
            for t in range(3):
                if t == a or hi[t] == lo[t]:
                    continue
                o = 3 - a - t
                for plane in (lo[a], hi[a] + 1):
                    blo, bhi = [0, 0, 0], [0, 0, 0]
                    blo[a] = bhi[a] = plane
                    blo[t], bhi[t] = lo[t], hi[t] - 1
                    blo[o], bhi[o] = lo[o], hi[o]
                    for e in _box_nodes(blo, bhi):
                        if (t, *e) not in self.sheet_edges:
                            m.zero_edges(0, t, e, e)
        f = self.file.signal
        nyq = f.nyquist_frequency()
        parallel = not series
        use = (not parallel) or (c is None and ind is not None)
        omega = 2.0 * math.pi * nyq if (use and nyq) else 0.0
        hi_node = list(hi)
        hi_node[a] += 1
        m.add_lumped_openems(a, lo, hi_node, r=r or 0.0, l=ind or 0.0, c=c or 0.0, series=series, omega=omega,
                             explicit=parallel)
        self.inductor_edges = getattr(self, "inductor_edges", set()) | {(a, *e) for e in edges}

    def _sheets(self, m):
        """openEMS's conducting sheets (emulate, src/compile/openems_sheet.rs:
        300-500): every in-plane E edge of a flat Box primitive on a mesh
        plane whose midpoint the sheet holds and wins (priority among
        materials, metal and sheets; lumped elements do not count) becomes a
        sheet edge, unless it lies on an outer mesh plane (left to the
        boundary). An edge in the first cell of its own axis, or with a node
        coordinate on a line that an absorbing boundary claims (Mur: the
        first and last two lines, PML_n: n + 1), is PEC. Its width is the
        dual edge across it at its start node, half of it on a border edge
        (one of the two neighbouring cells across it, at the start node,
        not held by a sheet, or the first cell of that axis, or in the
        boundary's lines); its circuit (openems_sheet.edge_circuit at the
        bin of the sheet's σ, t at the excitation's frequency) replaces the
        edge's medium, its two branches become sheet-branch poles. The time
        step was fixed before (openEMS's ignores the sheets)."""
        from . import openems_sheet as OS
        f = self.file
        sheets = [p for p in f.props if p.kind == "ConductingSheet"]
        if not sheets:
            return
        n, lines, dt = self.nodes, f.lines, self.dt
        freq = OS.sheet_frequency(f.signal, f.f_max)

        def reach(face):
            k, c = f.faces[face]
            return 1 if k == MUR_FACE else (int(c) if k == PML_FACE else 0)

        region = [(reach(2 * a), n[a] - 1 - reach(2 * a + 1)) for a in range(3)]

        def in_region(a, i):
            return i > 0 and (i <= region[a][0] or i >= region[a][1])

        def sheet_at(name, pt):
            w = self._winner(pt)
            return w is not None and w.kind == "ConductingSheet" and (not name or w.name == name)

        done = set()
        for p in sheets:
            sigma, th = _f(p.attrs.get("Conductivity")), _f(p.attrs.get("Thickness"))
            if not (sigma is not None and th is not None and math.isfinite(sigma) and sigma > 0
                    and math.isfinite(th) and th > 0):
                self.warnings.append(f"conducting sheet {p.name!r}: needs Conductivity > 0 and Thickness > 0; "
                                     "ignored")
                continue
            row = OS.TABLE[OS.bin_index(sigma, th, freq)]
            for b in p.boxes:
                if not (isinstance(b, Box) or (isinstance(b, LinPoly) and b.length == 0.0)):
                    raise NotImplementedError(f"conducting sheet {p.name!r}: primitives other than boxes and "
                                              "polygons")
                lo = [min(b.p1[q], b.p2[q]) for q in range(3)]
                hi = [max(b.p1[q], b.p2[q]) for q in range(3)]
                flat = [b.normal] if isinstance(b, LinPoly) else [q for q in range(3) if hi[q] == lo[q]]
                if len(flat) != 1:
                    raise NotImplementedError(f"conducting sheet {p.name!r}: a box that is not flat along one "
                                              "axis")
                nrm = flat[0]
                plane = [i for i, x in enumerate(lines[nrm]) if x == lo[nrm]]
                if not plane:
                    raise NotImplementedError(f"conducting sheet {p.name!r}: off the mesh planes")
                for d in range(3):
                    if d == nrm:
                        continue
                    t = 3 - d - nrm
                    along = [i for i in range(n[d] - 1)
                             if self._inside_prim(0.5 * (lines[d][i] + lines[d][i + 1]), lo[d], hi[d])]
                    across = [i for i in range(n[t]) if self._inside_prim(lines[t][i], lo[t], hi[t])]
                    for i_d in along:
                        for i_t in across:
                            node = [0, 0, 0]
                            node[d], node[t], node[nrm] = i_d, i_t, plane[0]
                            node = tuple(node)
                            if (d, node) in done:
                                continue
                            done.add((d, node))
                            if any(a != d and (node[a] == 0 or node[a] + 1 == n[a]) for a in range(3)):
                                continue
                            mid = [lines[q][node[q]] for q in range(3)]
                            mid[d] = 0.5 * (lines[d][node[d]] + lines[d][node[d] + 1])
                            if not sheet_at(p.name, mid):
                                continue

                            def holds(c):
                                pt = list(mid)
                                pt[d] = lines[d][node[d]]
                                pt[t] = 0.5 * (lines[t][c] + lines[t][c + 1])
                                return c != 0 and not in_region(t, c) and sheet_at("", pt)

                            interior = holds(node[t] - 1) and holds(node[t])
                            if node[d] == 0 or any(in_region(q, node[q]) for q in (d, t, nrm)):
                                m.zero_edges(0, d, node, node)
                                continue
                            dual = self.model_dual(t, node[t])
                            width = dual if interior else 0.5 * dual
                            branches, c_dt2, g_e = OS.edge_circuit(sigma, th, self.model_delta(d, node[d]) / width,
                                                                   row)
                            m.set_edge_circuit(d, node, cap=c_dt2 * dt * dt, cond=g_e)
                            self.sheet_edges.add((d, *node))
                            self.sheet_branches.append((d, node, branches))

    def _winner(self, pt, sheets: bool = True):
        """The property holding point ``pt`` (drawing units) by openEMS's
        priority (closed bounds; at equal priority the one defined first),
        among materials, metal and (``sheets``) conducting sheets; None for
        the background."""
        best = None
        kinds = MATERIALS + ("Metal",) + (("ConductingSheet",) if sheets else ())
        for p in self.file.props:
            if p.kind not in kinds:
                continue
            for b in p.boxes:
                if bool(b.inside(pt[0], pt[1], pt[2], self.tol)):
                    key = (b.priority, -p.order)
                    if best is None or key > best[0]:
                        best = (key, p)
        return best[1] if best else None

    def _dispersive(self, m):
        """Lorentz, Drude and Debye poles the openEMS way (src/compile/
        dispersive.rs:1-130, 480-560): every E edge (H dual edge) gets the
        full poles of the dispersive property winning at its midpoint (the
        centre of the face it pierces), ω_p = 2π·f_plasma, ω_0 = 2π·f_Lor,
        γ = 1/τ, Debye Δε, τ as given, dropped below three time steps; all
        with openEMS's f32 arithmetic (OpenEmsPole with the edge's own
        capacitance or inductance, openEMS's Debye update on edges of Debye
        poles alone)."""
        from . import OPENEMS_POLES, Dispersive, Pole
        f = self.file
        disp = [p for p in f.props if p.kind in ("LorentzMaterial", "DebyeMaterial")]
        if not disp:
            if self.sheet_branches:
                d = Dispersive()
                self._sheet_poles(d)
                m.add_dispersive(d, OPENEMS_POLES)
            return
        lines, n = f.lines, self.nodes
        co = [m.coeff(lane) for lane in (3, 4, 5, 9, 10, 11)]
        d = Dispersive()
        count = 0
        for field_ in (0, 1):
            for a in range(3):
                b, c = (a + 1) % 3, (a + 2) % 3
                # Candidate nodes: inside the dispersive boxes' bounding box.
                lo = [min(min(bx.p1[q], bx.p2[q]) for p in disp for bx in p.boxes) for q in range(3)]
                hi = [max(max(bx.p1[q], bx.p2[q]) for p in disp for bx in p.boxes) for q in range(3)]
                rng = []
                for q in range(3):
                    along = (q == a) == (field_ == 0)
                    last = n[q] - 1 if along else n[q]
                    rng.append([i for i in range(last)
                                if (along and lines[q][i + 1] >= lo[q] - 1e-9 and lines[q][i] <= hi[q] + 1e-9)
                                or (not along and lo[q] - 1e-9 <= lines[q][i] <= hi[q] + 1e-9)
                                or (not along and field_ == 1 and False)])
                if field_ == 1:
                    # H dual edge along a through node: midpoint at the node
                    # line along a, cell centres across.
                    rng = [([i for i in range(n[q]) if lo[q] - 1e-9 <= lines[q][i] <= hi[q] + 1e-9] if q == a else
                            [i for i in range(n[q] - 1) if lines[q][i + 1] >= lo[q] - 1e-9 and lines[q][i] <= hi[q] + 1e-9])
                           for q in range(3)]
                for i in rng[0]:
                    for j in rng[1]:
                        for k in rng[2]:
                            node = (i, j, k)
                            if field_ == 0:
                                if node[a] + 1 >= n[a] or co[a][node] == 0.0:
                                    continue
                                pt = [0.5 * (lines[q][node[q]] + lines[q][node[q] + 1]) if q == a else lines[q][node[q]]
                                      for q in range(3)]
                            else:
                                if node[b] + 1 >= n[b] or node[c] + 1 >= n[c] or co[3 + a][node] == 0.0:
                                    continue
                                pt = [lines[q][node[q]] if q == a else 0.5 * (lines[q][node[q]] + lines[q][node[q] + 1])
                                      for q in range(3)]
                            w = self._winner(pt)
                            if w is None or w.kind not in ("LorentzMaterial", "DebyeMaterial"):
                                continue
                            if field_ == 0 and (a, *node) in getattr(self, "inductor_edges", ()):
                                raise NotImplementedError("poles on the edges of a lumped element with an "
                                                          "inductor or in series (openEMS corrects them after "
                                                          "the element)")
                            for pole in self._poles(w, field_, a, 1.0, pt):
                                d.add_edge(field_, a, node, pole)
                                count += 1
        count += self._sheet_poles(d)
        if count:
            m.add_dispersive(d, OPENEMS_POLES)

    def _sheet_poles(self, d) -> int:
        """The conducting-sheet branches as sheet-branch poles of their
        edges (the reference's OpenEmsSheetBranches: the same f32 update)."""
        from . import Pole
        for a, node, branches in self.sheet_branches:
            for ind, res in branches:
                d.add_edge(0, a, node, Pole.sheet_branch(ind, res))
        return 2 * len(self.sheet_branches)

    def _poles(self, p, field_, a, inf, pt=None):
        from . import Pole
        iso = p.attrs.get("Isotropy", "1") != "0"
        order = int(float(p.attrs.get("Order", "1")))
        pre = "Epsilon" if field_ == 0 else "Mue"
        out = []
        for q in range(1, order + 1):
            def get(name, q=q):
                # "<name>_<order>", or for the first order also "<name>".
                v = p.prop.get(f"{pre}{name}_{q}")
                key = f"{pre}{name}_{q}"
                if v is None and q == 1:
                    v = p.prop.get(f"{pre}{name}")
                    key = f"{pre}{name}"
                x = _vec3(v, 0.0, iso)[a]
                # A weighting function of the parameter, at the edge midpoint.
                wf = p.weight.get(key) or (p.weight.get(f"{pre}{name}") if q == 1 else None)
                if wf and wf[a] is not None and pt is not None:
                    x *= float(wf[a].evaluate(x=pt[0], y=pt[1], z=pt[2]))
                return x

            if p.kind == "DebyeMaterial":
                if field_ == 1:
                    continue
                de, tau = get("Delta"), get("RelaxTime")
                if de != 0.0 and tau >= 3.0 * self.dt:
                    out.append(Pole.debye(de, tau))
                continue
            fp, fl, tau = get("PlasmaFrequency"), get("LorPoleFrequency"), get("RelaxTime")
            gamma = 1.0 / tau if tau > 0.0 else 0.0
            wp = TWO_PI * fp * math.sqrt(max(inf, 0.0))
            if wp == 0.0:
                continue
            out.append(Pole.drude(wp, gamma) if fl == 0.0 else Pole.lorentz(wp, TWO_PI * fl, gamma))
        return out

    @staticmethod
    def _material(m, prop, isotropic=True):
        eps = _vec3(prop.get("Epsilon"), 1.0, isotropic)
        mu = _vec3(prop.get("Mue"), 1.0, isotropic)
        kap = _vec3(prop.get("Kappa"), 0.0, isotropic)
        sig = _vec3(prop.get("Sigma"), 0.0, isotropic)
        return m.material(eps_r=tuple(eps), mu_r=tuple(mu), kappa=tuple(kap), sigma_m=tuple(sig))

    def _lossy(self):
        f = self.file
        props = [p.prop for p in f.props if p.kind in MATERIALS] + ([f.background] if f.background else [])
        return any(any(float(x) != 0.0 for x in (pr.get(k) or "0").split(","))
                   for pr in props for k in ("Kappa", "Sigma"))

    def _pmc_half_cell(self, m):
        """openEMS's PMC (src/compile/mod.rs:1556-1626): the tangential H of
        the dual layer next to the face, the tangential E and the normal H
        on the face are never updated, except a lumped element's E edges
        and the H dual edge of the same direction and node as a
        conducting-sheet edge or an edge of a lumped element with an
        inductor or in series (src/compile/mod.rs:1180-1197)."""
        n = self.nodes
        keep = {(a, tuple(e)) for a, *e in self.sheet_edges | self.branch_edges}
        keep_e = {(a, tuple(e)) for a, *e in self.lumped_edges}
        for face, (k, _) in enumerate(self.file.faces):
            if k != PMC_FACE:
                continue
            t, is_max = face // 2, face % 2 == 1
            h_layer, e_layer = (n[t] - 2, n[t] - 1) if is_max else (0, 0)
            for a in range(3):
                todo = [(1, e_layer)] if a == t else [(1, h_layer), (0, e_layer)]
                for field_, layer in todo:
                    lo, hi = [0, 0, 0], [n[0] - 1, n[1] - 1, n[2] - 1]
                    lo[t] = hi[t] = layer
                    kept = [e for (ka, e) in (keep if field_ == 1 else keep_e) if ka == a and e[t] == layer]
                    if not kept:
                        m.zero_edges(field_, a, lo, hi)
                        continue
                    # Row by row along the last in-plane axis, around the kept edges.
                    u, w = [q for q in range(3) if q != t]
                    for iu in range(n[u]):
                        skip = sorted(e[w] for e in kept if e[u] == iu)
                        start = 0
                        for stop in skip + [n[w]]:
                            if stop > start:
                                blo, bhi = list(lo), list(hi)
                                blo[u] = bhi[u] = iu
                                blo[w], bhi[w] = start, stop - 1
                                m.zero_edges(field_, a, blo, bhi)
                            start = stop + 1

    def _excitation_winner(self, pt):
        """The excitation property that owns point ``pt``: the highest
        priority containing it, ties to the one defined first, disabled
        ones included (excitation_priority, src/compile/openems.rs:
        245-300)."""
        best = None
        for p in self.file.props:
            if p.kind != "Excitation":
                continue
            for b in p.boxes:
                inside = (all(self._inside_prim(pt[q], min(b.p1[q], b.p2[q]), max(b.p1[q], b.p2[q])) for q in range(3))
                          if isinstance(b, Box) else bool(b.inside(pt[0], pt[1], pt[2], self.tol)))
                if inside:
                    key = (b.priority, -p.order)
                    if best is None or key > best[0]:
                        best = (key, p)
        return best[1] if best else None

    def _excitation_edges(self):
        """(E?, axis, node, weight per unit amplitude, property) of every
        driven edge: E edges whose both nodes lie in the closed box (whose
        midpoint lies in a sphere, cylinder or shell), H dual edges whose
        midpoint does; weight = Excite × (dual) edge length.
        openEMS gives each edge to one excitation: the one owning the edge
        midpoint (E types) or the dual edge's (H types)."""
        out = []
        f = self.file
        n = self.nodes
        lines = f.lines
        for p in f.props:
            if p.kind != "Excitation" or p.attrs.get("Enabled", "1") == "0":
                continue
            typ = int(float(p.attrs.get("Type", "0")))
            if typ not in (0, 1, 2, 3):
                raise NotImplementedError(f"excitation type {typ}")
            e_type = typ in (0, 1)
            exc = _vec3(p.attrs.get("Excite"), 0.0, isotropic=False)
            for b in p.boxes:
                lo = [min(b.p1[a], b.p2[a]) for a in range(3)]
                hi = [max(b.p1[a], b.p2[a]) for a in range(3)]
                for a in range(3):
                    if exc[a] == 0.0:
                        continue
                    rng = []
                    box = isinstance(b, Box)
                    for q in range(3):
                        if e_type and not box:
                            # A round primitive: the candidates of its
                            # bounding box, then both nodes inside it.
                            pts = [i for i in range(n[q] - (1 if q == a else 0))
                                   if lines[q][i + (1 if q == a else 0)] >= lo[q] - self.tol
                                   and lines[q][i] <= hi[q] + self.tol]
                        elif e_type:
                            pts = [i for i in range(n[q] - (1 if q == a else 0))
                                   if self._inside_prim(lines[q][i], lo[q], hi[q])
                                   and (q != a or self._inside_prim(lines[q][i + 1], lo[q], hi[q]))]
                        else:
                            if q == a:
                                pts = [i for i in range(n[q]) if self._inside_prim(lines[q][i], lo[q], hi[q])]
                            else:
                                pts = [i for i in range(n[q] - 1)
                                       if self._inside_prim(0.5 * (lines[q][i] + lines[q][i + 1]), lo[q], hi[q])]
                        rng.append(pts)
                    for i in rng[0]:
                        for j in rng[1]:
                            for k in rng[2]:
                                node = (i, j, k)
                                if e_type and not box:
                                    pm = [lines[q][node[q]] for q in range(3)]
                                    pm[a] = 0.5 * (lines[a][node[a]] + lines[a][node[a] + 1])
                                    if not b.inside(*pm, self.tol):
                                        continue
                                if e_type:
                                    length = self.model_delta(a, node[a])
                                else:
                                    length = self.model_dual(a, node[a])
                                mid = [0.5 * (lines[q][node[q]] + lines[q][node[q] + 1])
                                       if ((q == a) == e_type) and node[q] + 1 < n[q] else lines[q][node[q]]
                                       for q in range(3)]
                                if self._excitation_winner(mid) is not p:
                                    continue
                                wx = p.weight.get("Excite", [None] * 3)[a]
                                g = float(wx.evaluate(x=mid[0], y=mid[1], z=mid[2])) if wx is not None else 1.0
                                out.append((e_type, typ, a, node, exc[a] * g * length, p))
        return out

    def model_delta(self, a, i):
        return float(self.lines_m[a][i + 1] - self.lines_m[a][i])

    def model_dual(self, a, i):
        v = self.lines_m[a]
        lo = v[i] - v[i - 1] if i > 0 else 0.0
        hi = v[i + 1] - v[i] if i + 1 < len(v) else 0.0
        return float(0.5 * (lo + hi))

    def _mur(self, m):
        f = self.file
        faces = {fc: f.mur_velocity for fc, (k, _) in enumerate(f.faces) if k == MUR_FACE}
        if not faces:
            return
        from . import MUR_COUNT_ENERGY, MUR_OPENEMS_CORNERS, MUR_OPENEMS_ORDER
        hold = None
        if f.signal.kind == 0:
            n = self.nodes
            held = set()
            for e_type, _, a, node, _, _ in self.excited:
                if not e_type:
                    continue
                for fc in faces:
                    fa = fc // 2
                    plane = n[fa] - 1 if fc % 2 else 0
                    if fa != a and node[fa] == plane:
                        held.add(fc)
            if held:
                steps = int(math.floor(2.0 * f.signal.delay / self.dt)) + 1
                hold = {fc: steps + 10 for fc in held}
        self._mur_media(m, [fc for fc, v in faces.items() if v is None])
        m.add_mur(faces, hold=hold, flags=MUR_COUNT_ENERGY | MUR_OPENEMS_CORNERS | MUR_OPENEMS_ORDER)

    def _refuse_poles_beside_mur(self, m):
        """openEMS's Mur faces take the interior neighbours before the
        poles' correction of their update (src/compile/mod.rs:1258-1263),
        an interplay not restated here: E pole edges on a Mur face plane or
        on the plane inside it (tangential to the face) are refused."""
        from . import OP_POLES, EngineDesc, OpEntry, PolesTable
        mur = [fc for fc, (k, _) in enumerate(self.file.faces) if k == MUR_FACE]
        d = EngineDesc.from_address(m.desc)
        if not mur or not d.n_ops:
            return
        n = self.nodes
        for o in (OpEntry * d.n_ops).from_address(d.ops):
            if o.kind != OP_POLES:
                continue
            pe = PolesTable.from_address(o.table).electric
            ne = int(pe.n_edges)
            if not ne:
                continue
            flat = np.ctypeslib.as_array((ctypes.c_uint64 * ne).from_address(pe.node)).astype(np.int64)
            axis = np.ctypeslib.as_array((ctypes.c_uint8 * ne).from_address(pe.axis))
            ijk = (flat // (n[1] * n[2]), (flat // n[2]) % n[1], flat % n[2])
            for fc in mur:
                fa = fc // 2
                plane = n[fa] - 1 if fc % 2 else 0
                if np.any((np.abs(ijk[fa] - plane) <= 1) & (axis != fa)):
                    raise NotImplementedError("dispersive media on or beside a Mur face (openEMS's Mur reads the "
                                              "interior neighbours before the poles' correction)")

    def _absorbing_sheets(self, m):
        """csx ``AbsorbingBC`` properties (src/compile/mod.rs:106-125,
        1999-2080, 1424-1432): every box, snapped to the nearest mesh lines,
        must be flat along exactly one axis (the sheet normal; volumes,
        lines and points are ignored with a warning); NormalSignPositive
        is the sign of the normal into the region the sheet terminates, so
        the sheet absorbs waves along the opposite sign; PhaseVelocity > 0
        as given, 0 the local medium velocity (negative or not finite: the
        local one, with a warning); AbsorbingBoundaryType other than 0
        (MUR_1ST) runs as first-order Mur with a warning. Installed with
        openEMS's order (``Model.add_absorbing_sheet``)."""
        f = self.file
        lines = f.lines
        for p in f.props:
            if p.kind != "AbsorbingBC":
                continue
            if not p.boxes:
                self.warnings.append(f"AbsorbingBC {p.name!r}: no primitive; ignored")
                continue
            typ = int(float(p.attrs.get("AbsorbingBoundaryType", "0")))
            if typ != 0:
                self.warnings.append(f"AbsorbingBC {p.name!r}: AbsorbingBoundaryType {typ} not implemented; "
                                     "first-order Mur (MUR_1ST) used")
            v = _f(p.attrs.get("PhaseVelocity"), 0.0)
            if not (math.isfinite(v) and v > 0.0):
                if v != 0.0:
                    self.warnings.append(f"AbsorbingBC {p.name!r}: PhaseVelocity {v} invalid; local medium "
                                         "velocity used")
                v = 0.0
            positive = p.attrs.get("NormalSignPositive", "0") in ("0", "false", "False")
            for b in p.boxes:
                if not isinstance(b, Box):
                    raise NotImplementedError(f"AbsorbingBC {p.name!r}: primitives other than boxes")
                snap = [(int(np.argmin(np.abs(np.asarray(lines[q]) - b.p1[q]))),
                         int(np.argmin(np.abs(np.asarray(lines[q]) - b.p2[q])))) for q in range(3)]
                start = [min(x) for x in snap]
                stop = [max(x) for x in snap]
                flat = [q for q in range(3) if start[q] == stop[q]]
                if len(flat) != 1:
                    what = "a volume" if not flat else "a line or point"
                    self.warnings.append(f"AbsorbingBC {p.name!r}: primitive is {what} on the mesh, not a sheet; "
                                         "ignored")
                    continue
                d = flat[0]
                if b.p1[d] != b.p2[d]:
                    self.warnings.append(f"AbsorbingBC {p.name!r}: primitive has a thickness along "
                                         f"{'xyz'[d]}; flattened onto mesh plane {start[d]}")
                m.add_absorbing_sheet(d, start[d], positive, start, stop, velocity=v, openems_order=True)

    def _mur_media(self, m, faces):
        """The medium of each edge of a Mur face without a phase velocity
        the openEMS way (mur_point_media, src/compile/mod.rs:1641-1699): the
        material at one point, the edge's start node across and the middle
        of the boundary cell along the normal (closed, metal not counted),
        ε along the edge and μ along the other tangential axis,
        v = c0/√(εμ)."""
        f = self.file
        n = self.nodes
        lines = f.lines
        mats = [p for p in f.props if p.kind in MATERIALS]
        for fc in faces:
            a = fc // 2
            plane, inner = (n[a] - 1, n[a] - 2) if fc % 2 else (0, 1)
            mid = 0.5 * (lines[a][plane] + lines[a][inner])
            u, w = [q for q in range(3) if q != a]
            for t in (u, w):
                o = w if t == u else u
                v = np.zeros((n[u], n[w]))
                for pu in range(n[u]):
                    for pw in range(n[w]):
                        node = [0, 0, 0]
                        node[a], node[u], node[w] = plane, pu, pw
                        if node[t] + 1 >= n[t]:
                            continue
                        pt = [lines[q][node[q]] for q in range(3)]
                        pt[a] = mid
                        best = None
                        for p in mats:
                            for b in p.boxes:
                                if bool(b.inside(pt[0], pt[1], pt[2], self.tol)):
                                    key = (b.priority, -p.order)
                                    if best is None or key > best[0]:
                                        best = (key, p)
                        prop = best[1].prop if best else f.background
                        iso = best[1].attrs.get("Isotropy", "1") != "0" if best else True
                        eps = _vec3(prop.get("Epsilon"), 1.0, iso)[t] if prop else 1.0
                        mu = _vec3(prop.get("Mue"), 1.0, iso)[o] if prop else 1.0
                        wt = best[1].weight if best else {}
                        at = dict(zip("xyz", pt))
                        if wt.get("Epsilon") and wt["Epsilon"][t] is not None:
                            eps *= float(wt["Epsilon"][t].evaluate(**at))
                        if wt.get("Mue") and wt["Mue"][o] is not None:
                            mu *= float(wt["Mue"][o].evaluate(**at))
                        v[pu, pw] = C0 / math.sqrt(eps * mu)
                m.set_mur_media(fc, t, v)

    def _excitations(self, m):
        from . import HARD_E, HARD_H, SOFT_E, SOFT_H
        f, dt, steps = self.file, self.dt, self.steps + 1
        kinds = {0: SOFT_E, 1: HARD_E, 2: SOFT_H, 3: HARD_H}
        by_prop = {}
        for e_type, typ, a, node, w, p in self.excited:
            by_prop.setdefault(p.order, (typ, p, []))[2].append((a, node, w))
        for order in sorted(by_prop):
            typ0, p, all_edges = by_prop[order]
            groups = [(typ0, all_edges)]
            on = [e for e in all_edges if (e[0], *e[1]) in self.sheet_edges] if typ0 == 1 else []
            if on:
                # openEMS's sheet edges keep their update under a hard E
                # source: it adds to them as a soft one (src/sim/map.rs:
                # 688-700, 773-792).
                self.warnings.append(f"excitation {p.name!r}: hard E source on {len(on)} conducting-sheet edge(s); "
                                     "excited as a soft source there (openEMS's sheet keeps its update)")
                groups = [(0, on), (1, [e for e in all_edges if (e[0], *e[1]) not in self.sheet_edges])]
            for typ, edges in groups:
                if not edges:
                    continue
                kind = kinds[typ]
                hard = typ in (1, 3)
                lag = dt if hard else 0.5 * dt
                delay = _f(p.attrs.get("Delay"), 0.0)
                shift = lag + (math.floor(delay / dt) if delay > 0 else 0) * dt
                # The kind's sample time of step n (SourceKind).
                t_of = {SOFT_E: lambda s: (s + 0.5) * dt, HARD_E: lambda s: (s + 1.0) * dt,
                        SOFT_H: lambda s: s * dt, HARD_H: lambda s: (s + 0.5) * dt}[kind]
                amp = np.zeros(steps)
                for s in range(steps):
                    tau = t_of(s) - shift
                    amp[s] = 0.0 if tau < -0.25 * dt else f.signal.value(tau, dt)
                m.add_source_table(kind, edges, amp)
                if kind == HARD_E:
                    # openEMS's hard E source edges have no update of their
                    # own: the operators acting after the update (its Mur
                    # faces) read them as 0 before the source writes
                    # (src/sim/map.rs:1007-1027). Not in its PML layers,
                    # whose update is completed there.
                    in_pml = set()
                    if self.upml_op is not None:
                        ax, nodes, _ = m.upml_table(self.upml_op)[0]
                        in_pml = {(int(a), *map(int, nd)) for a, nd in zip(ax, nodes)}
                    for a, node, _ in edges:
                        if (a, *node) not in in_pml:
                            m.zero_edges(0, a, node, node)
                if typ in (2, 3):
                    self.h_sources.append((typ == 3, edges, amp.astype(np.float32)))

    def _mode_probe(self, m, p, typ, weight, os_, window):
        """A waveguide (mode-matching) probe with openEMS's sampling
        (src/compile/mode.rs:1-60, 147-258, 386-540): the box snapped to
        the nearest lines, its normal NormDir or its flat axis; samples at
        the box's nodes (voltage, type 10) or at the centres of its cells
        (current, type 11), never on the outermost mesh lines; the mode
        function ModeFunctionX/Y/Z (drawing units) at each sample,
        normalised by the probe itself, V = w·Σ E_t·f·A/√(Σ|f_t|²·A) with
        E_t at a node the linear interpolation of the two edges along t
        through it, I = w·Σ H_t·f·A/√(Σ|f_t|²·A) with H_t at the cell's
        lower corner (the mean of the two dual edges beside it, each the
        mean of the H planes k ± ½). The value is one probe; each sample's
        two field components are probes too, for the mode purity
        w·(Σ A·F·f)²/(Σ A·|F|²·Σ A·|f|²)."""
        from . import CURRENT, VOLTAGE
        f, n = self.file, self.nodes
        lines, lm, unit = f.lines, self.lines_m, f.unit
        funcs = []
        for c in "XYZ":
            src = p.user.get(f"ModeFunction{c}", "0")
            funcs.append(Expression(src, ("x", "y", "z")))
        b0 = p.boxes[0]
        near = lambda q, v: int(np.argmin(np.abs(np.asarray(lines[q]) - v)))  # noqa: E731
        start = [near(q, b0.p1[q]) for q in range(3)]
        stop = [near(q, b0.p2[q]) for q in range(3)]
        norm = p.attrs.get("NormDir")
        if norm is not None:
            nn = int(float(norm))
        else:
            flat = [q for q in range(3) if start[q] == stop[q]]
            if len(flat) != 1:
                self.warnings.append(f"waveguide probe {p.name!r}: no normal direction; ignored")
                return
            nn = flat[0]
        k = start[nn]
        lo = [min(start[q], stop[q]) for q in range(3)]
        hi = [max(start[q], stop[q]) for q in range(3)]
        current = typ == 11
        ta, tb = [q for q in range(3) if q != nn]
        delta = lambda q, i: float(lm[q][i + 1] - lm[q][i])  # noqa: E731

        def rng(d):
            top = hi[d] - 1 if current else hi[d]
            return range(max(lo[d], 1), min(top, n[d] - 2) + 1)

        samples = []
        for i in rng(ta):
            for j in rng(tb):
                pt = [0.0] * 3
                pt[nn] = float(lm[nn][k])
                if current:
                    pt[ta] = 0.5 * float(lm[ta][i] + lm[ta][i + 1])
                    pt[tb] = 0.5 * float(lm[tb][j] + lm[tb][j + 1])
                    area = delta(ta, i) * delta(tb, j)
                else:
                    pt[ta], pt[tb] = float(lm[ta][i]), float(lm[tb][j])
                    area = self.model_dual(ta, i) * self.model_dual(tb, j)
                env = dict(x=pt[0] / unit, y=pt[1] / unit, z=pt[2] / unit)
                samples.append(((i, j), (float(funcs[ta].evaluate(**env)), float(funcs[tb].evaluate(**env))), area))
        ra, rb = rng(ta), rng(tb)
        llo, lhi = [k] * 3, [k] * 3
        if len(ra) and len(rb):
            llo[ta], lhi[ta], llo[tb], lhi[tb] = ra[0], ra[-1], rb[0], rb[-1]
        at = lambda idx: tuple(float(lm[q][idx[q]]) for q in range(3))  # noqa: E731
        location = ((at(llo), llo), (at(lhi), lhi))
        q_kind = CURRENT if current else VOLTAGE
        norm2 = sum((fv[0] ** 2 + fv[1] ** 2) * area for _, fv, area in samples)
        kind = "current_mode" if current else "voltage_mode"
        if not (norm2 > 0.0 and math.isfinite(norm2)):
            self.warnings.append(f"waveguide probe {p.name!r}: the mode function is zero on the probe plane; "
                                 "it reads 0")
            kk = m.add_probe(q_kind, [(0, (0, 0, 0), 0.0)])
            self.probes.append(ProbeSpec(p.name, kind, [kk], location, p.fd, os_, *window, (weight, [])))
            return
        scale = 1.0 / math.sqrt(norm2)
        planes = ([(k - 1, 0.5), (k, 0.5)] if (k > 0 and k + 1 < n[nn]) else
                  [(k - 1, 1.0)] if k > 0 else [(k, 1.0)] if k + 1 < n[nn] else [])
        entries, purity = [], []
        for (i, j), fv, area in samples:
            w = area * scale
            fields = [[], []]
            for c, (t, o) in enumerate(((ta, tb), (tb, ta))):
                it, io = (i, j) if c == 0 else (j, i)
                fc = fv[c] * w
                node = [0, 0, 0]
                node[nn], node[o] = k, io
                if current:
                    for oc in (io - 1, io):
                        for kp, wp in planes:
                            node[t], node[o], node[nn] = it, oc, kp
                            coef = 0.5 * wp / self.model_dual(t, it)
                            fields[c].append((t, tuple(node), coef))
                            if fc != 0.0 and math.isfinite(fc * coef):
                                entries.append((t, tuple(node), fc * 0.5 * wp / self.model_dual(t, it)))
                else:
                    dl, dh = delta(t, it - 1), delta(t, it)
                    wl, wh = dh / (dl + dh), dl / (dl + dh)
                    for idx, cw in ((it - 1, wl / dl), (it, wh / dh)):
                        node[t] = idx
                        fields[c].append((t, tuple(node), cw))
                        if fc != 0.0 and math.isfinite(fc * cw):
                            entries.append((t, tuple(node), fc * cw))
            ops = tuple(m.add_probe(q_kind, fl) for fl in fields)
            purity.append((area, fv, ops))
        kk = m.add_probe(q_kind, [(a, nd, v * weight) for a, nd, v in entries] or [(0, (0, 0, 0), 0.0)])
        self.probes.append(ProbeSpec(p.name, kind, [kk], location, p.fd, os_, *window, (weight, purity)))

    def _probes(self, m):
        from . import CURRENT, VOLTAGE
        f = self.file
        n = self.nodes
        lines = f.lines
        at = lambda idx: tuple(float(self.lines_m[a][idx[a]]) for a in range(3))  # noqa: E731
        for p in f.props:
            if p.kind != "ProbeBox" or not p.boxes:
                continue
            typ = int(float(p.attrs.get("Type", "0")))
            weight = float(p.attrs.get("Weight", "1"))
            c0, c1 = p.boxes[0].p1, p.boxes[0].p2
            window = (_f(p.attrs.get("StartTime"), 0.0), _f(p.attrs.get("StopTime"), 0.0))
            os_attr = p.attrs.get("OverSampling")
            os_ = int(float(os_attr)) if os_attr is not None else None
            if typ in (10, 11):
                self._mode_probe(m, p, typ, weight, os_, window)
                continue
            if typ not in (0, 1, 2, 3):
                self.warnings.append(f"probe {p.name!r}: type {typ} not supported; ignored")
                continue
            extent = [a for a in range(3) if c0[a] != c1[a]]
            norm = p.attrs.get("NormDir")
            norm = int(float(norm)) if norm is not None else None
            if typ == 0 and len(extent) != 1:
                self.warnings.append(f"probe {p.name!r}: its box is not a line; ignored, as openEMS does")
                continue
            if typ == 1 and ((norm is not None and norm in extent) or (norm is None and len(extent) == 3)):
                self.warnings.append(f"probe {p.name!r}: not flat along its normal; ignored, as openEMS does")
                continue
            prim = lambda c: [snap_lower(lines[a], c[a]) for a in range(3)]  # noqa: E731
            dual = lambda c: [snap_cell(lines[a], c[a]) for a in range(3)]  # noqa: E731
            if typ == 0:
                start, stop = prim(c0), prim(c1)
                path = voltage_path(start, stop)
                k = m.add_probe(VOLTAGE, [(a, nd, w * weight) for a, nd, w in path]) if path else \
                    m.add_probe(VOLTAGE, [(0, (0, 0, 0), 0.0)])
                self.probes.append(ProbeSpec(p.name, "voltage", [k], ((at(start), start), (at(stop), stop)),
                                             p.fd, os_, *window))
            elif typ == 1:
                start = [snap_lower(lines[a], c0[a]) for a in range(3)]
                stop = [snap_lower(lines[a], c1[a]) for a in range(3)]
                if norm is None:
                    flat = [a for a in range(3) if start[a] == stop[a]]
                    if len(flat) != 1:
                        self.warnings.append(f"probe {p.name!r}: no normal direction; ignored")
                        continue
                    norm = flat[0]
                nn = norm
                crossed = [False] * 3
                for a in range(3):
                    if a == nn:
                        continue
                    r0, r1 = c0[a], c1[a]
                    lo = snap_upper(lines[a], min(r0, r1))
                    hi = snap_lower(lines[a], max(r0, r1))
                    crossed[a] = lo > hi
                    start[a], stop[a] = (lo, hi) if r0 <= r1 else (hi, lo)
                flat_layer = dual(c0)[nn] if start[nn] == stop[nn] else None
                lo = [min(start[a], stop[a]) for a in range(3)]
                hi = [max(start[a], stop[a]) for a in range(3)]
                if flat_layer is not None:
                    layer = min(flat_layer, n[nn] - 2)
                elif lo[nn] == hi[nn]:
                    layer = min(lo[nn], n[nn] - 2)
                else:
                    layer = lo[nn] + (hi[nn] - lo[nn] - 1) // 2
                sign = 1.0 if start[nn] <= stop[nn] else -1.0
                entries = [(a, nd, -w * sign) for a, nd, w in loop_entries(nn, lo, hi, layer)]
                entries = openems_loop_order(entries, nn, start, stop)
                llo, lhi = [0, 0, 0], [0, 0, 0]
                for d in range(3):
                    if d == nn:
                        llo[d] = lhi[d] = layer
                    else:
                        a_, b_ = min(start[d], stop[d]), max(start[d], stop[d])
                        if crossed[d]:
                            a_, b_ = b_, a_
                        llo[d], lhi[d] = max(a_ - 1, 0), min(b_, max(n[d] - 2, 0))
                if any(crossed):
                    entries = []
                if entries:
                    k = m.add_probe(CURRENT, [(a, nd, w * weight) for a, nd, w in entries], f32_sum=True)
                else:
                    k = m.add_probe(CURRENT, [(0, (0, 0, 0), 0.0)])
                self.probes.append(ProbeSpec(p.name, "current", [k], ((at(llo), llo), (at(lhi), lhi)), p.fd, os_,
                                             *window))
            else:
                e = typ == 2
                idx = prim(c0) if e else dual(c0)
                loc = ((at(prim(c0)), prim(c0)), (at(prim(c1)), prim(c1))) if e else \
                    ((at(idx), idx), (at(dual(c1)), dual(c1)))
                ks = []
                for a in range(3):
                    ok = all((idx[b] + 1 < n[b]) if ((b == a) == e) else True for b in range(3))
                    length = 0.0
                    if ok:
                        length = self.model_delta(a, idx[a]) if e else self.model_dual(a, idx[a])
                    q = VOLTAGE if e else CURRENT
                    if ok and length > 0:
                        ks.append(m.add_probe(q, [(a, tuple(idx), weight / length)]))
                    else:
                        ks.append(m.add_probe(q, [(a, (0, 0, 0), 0.0)]))
                self.probes.append(ProbeSpec(p.name, "efield" if e else "hfield", ks, loc, p.fd, os_, *window))

    # -- running and output
    def energy(self, engine, step: int, curl_order: int = 1) -> float:
        """openEMS's energy measure of the engine's state
        (EnergyMeasure::OpenEms, src/engine/run.rs:66-76, kernel.rs:364-414,
        dump.rs:1735-1785): ε0·Σu² over the E edges but those on the three
        upper faces, plus μ0·Σ w·h² over the H dual edges with h the next H
        update evaluated from the state (the H sources of the next step
        included) and w = 4 on the outer planes normal to the edge."""
        n = self.nodes
        u = [engine.field(0, a).astype(np.float32) for a in range(3)]
        i = [engine.field(1, a).astype(np.float32) for a in range(3)]
        co = [self.model.coeff(lane) for lane in range(12)]
        we = sum(float(np.sum(np.square(u[a][:-1, :-1, :-1].astype(np.float64)))) for a in range(3))
        tiny = np.float32(np.finfo(np.float32).tiny)

        def fl(x):
            return np.where(np.abs(x) < tiny, np.float32(0.0), x).astype(np.float32)

        def upd(da, h, db, a, b, c, d):
            if curl_order:
                curl = fl(fl(fl(a - b) + d) - c)
                return fl(fl(da * h) - fl(db * curl))
            return fl(da * h - db * ((a - b) - (c - d)))

        z = np.zeros_like(u[0])
        sh = lambda x, ax: np.concatenate([x.take(range(1, x.shape[ax]), axis=ax),  # noqa: E731
                                           z.take([0], axis=ax)], axis=ax)
        hn = [upd(co[6], i[0], co[9], sh(u[2], 1), u[2], sh(u[1], 2), u[1]),
              upd(co[7], i[1], co[10], sh(u[0], 2), u[0], sh(u[2], 0), u[2]),
              upd(co[8], i[2], co[11], sh(u[1], 0), u[1], sh(u[0], 1), u[0])]
        for hard, edges, amp in self.h_sources:
            a_ = amp[step] if step < len(amp) else np.float32(0.0)
            for ax, node, w in edges:
                v = np.float32(np.float32(w) * a_)
                hn[ax][node] = v if hard else np.float32(hn[ax][node] + v)
        valid = [(slice(None), slice(0, n[1] - 1), slice(0, n[2] - 1)),
                 (slice(0, n[0] - 1), slice(None), slice(0, n[2] - 1)),
                 (slice(0, n[0] - 1), slice(0, n[1] - 1), slice(None))]
        wh = 0.0
        for a in range(3):
            x = hn[a].astype(np.float64) ** 2
            wgt = np.ones(n[a])
            wgt[0] = wgt[-1] = 4.0
            shape = [1, 1, 1]
            shape[a] = n[a]
            wh += float(np.sum((x * wgt.reshape(shape))[valid[a]]))
        from . import eps0, mu0
        w = eps0() * we + mu0() * wh
        if self.upml_op is not None and len(self.upml_h[0]):
            w += mu0() * self._upml_energy_correction(engine, u, co)
        return w

    def _upml_energy_correction(self, engine, u, co):
        """What openEMS's measure misses on the PML layers' H edges, whose
        look-ahead is the flux increment (upml.rs:466-506): Σ x² − inc² with
        inc = −db·(curl in the default order) and x its layer update."""
        ax, nodes, c = self.upml_h
        F, v = engine.upml_state(self.upml_op, 1, len(ax))
        tiny = np.float32(np.finfo(np.float32).tiny)

        def fl(x):
            return np.where(np.abs(x) < tiny, np.float32(0.0), x).astype(np.float32)

        i, j, k = nodes[:, 0], nodes[:, 1], nodes[:, 2]
        t = np.zeros(len(ax), dtype=np.float32)
        for a in range(3):
            sel = ax == a
            ii, jj, kk = i[sel], j[sel], k[sel]
            if a == 0:
                t[sel] = (u[2][ii, jj + 1, kk] - u[2][ii, jj, kk]) - (u[1][ii, jj, kk + 1] - u[1][ii, jj, kk])
            elif a == 1:
                t[sel] = (u[0][ii, jj, kk + 1] - u[0][ii, jj, kk]) - (u[2][ii + 1, jj, kk] - u[2][ii, jj, kk])
            else:
                t[sel] = (u[1][ii + 1, jj, kk] - u[1][ii, jj, kk]) - (u[0][ii, jj + 1, kk] - u[0][ii, jj, kk])
        db = np.array([co[9 + a][n_] for a, n_ in zip(ax, map(tuple, nodes))], dtype=np.float32)
        inc = fl(np.float32(0.0) * v - db * t)
        f1 = fl(fl(c[:, 0] * F) + inc)
        x = fl(fl(fl(c[:, 1] * v) - fl(c[:, 3] * F)) + fl(c[:, 2] * f1))
        return float(np.sum(x.astype(np.float64) ** 2 - inc.astype(np.float64) ** 2))

    def _drive(self, engine, curl_order) -> int:
        """The reference's run loop for files (src/engine/run.rs:424-540
        with check_after_interval, src/sim/mod.rs:910-930): openEMS's energy
        measure every Nyquist interval and once after half the Gaussian's
        length; stops when it falls below endCriteria times its maximum."""
        k = self.file.signal.nyquist_interval(self.dt)
        extra = None
        if self.file.signal.kind == 0:
            extra = self.file.signal.length(self.dt, self.steps) // 2
        steps, w_max = 0, 0.0
        self.stopped, self.last_ratio_db = False, None
        while steps < self.steps:
            regular = (steps // k + 1) * k
            nxt = extra if (extra is not None and steps < extra < regular) else regular
            nxt = min(nxt, self.steps)
            engine.run(nxt - steps)
            steps = nxt
            if steps % k and steps != extra:
                continue
            w = self.energy(engine, steps, curl_order)
            w_max = max(w_max, w)
            if not math.isfinite(w) or w < -1e-12 * w_max:
                self.warnings.append("diverged")
                break
            self.last_ratio_db = 10.0 * math.log10(w / w_max) if w > 0.0 and w_max > 0.0 else -math.inf
            if w_max > 0.0 and w / w_max < self.criterion:
                self.stopped = True
                break
        return steps

    @staticmethod
    def _purity(engine, p) -> np.ndarray:
        """The mode purity series of a waveguide probe (Probe::mode_purity,
        src/engine/probe.rs:314-330): w·(Σ A·F·f)²/(Σ A·|F|²·Σ A·|f|²) per
        sample, 0 where the field is 0."""
        weight, samples = p.purity
        n = len(engine.samples(p.ops[0]))
        if not samples:
            return np.zeros(n)
        dot = np.zeros(n)
        ff = np.zeros(n)
        mm = 0.0
        for area, fv, (ox, oy) in samples:
            fx, fy = np.asarray(engine.samples(ox)), np.asarray(engine.samples(oy))
            dot += area * (fx * fv[0] + fy * fv[1])
            ff += area * (fx * fx + fy * fy)
            mm += area * (fv[0] ** 2 + fv[1] ** 2)
        den = ff * mm
        with np.errstate(all="ignore"):
            return np.where(den > 0.0, weight * dot * dot / np.where(den > 0.0, den, 1.0), 0.0)

    def run(self, engine, curl_order: int = 1) -> "Results":
        """Runs ``engine`` (built on ``self.model``) to the end criterion or
        the run length, then one step more, whose H update gives the H-type
        probes' sample after the last step, and collects the probe series.
        ``curl_order`` 1 sums the curl in openEMS's order, as the reference
        does for files (its fields then equal openEMS's where the
        coefficients do), 0 in the engine's default order."""
        engine.set_curl_order(curl_order)
        self.stopped, self.last_ratio_db = False, None
        if self.criterion is None:
            engine.run(self.steps + 1)
            self.steps_run = self.steps
        else:
            self.steps_run = self._drive(engine, curl_order)
            engine.run(1)
        n = self.steps_run
        series = {}
        for p in self.probes:
            cols = [np.asarray(engine.samples(k)) for k in p.ops]
            if p.purity is not None:
                cols.append(self._purity(engine, p))
            v = np.stack(cols, axis=1)
            magnetic = p.kind in PF.MAGNETIC
            series[p.name] = v[: n + 1] if magnetic else v[:n]
        return Results(self, series)



@dataclass
class Results:
    setup: Setup
    series: dict

    def rows(self, p: ProbeSpec) -> list:
        """(step, time, values) of every sample of probe ``p`` in its
        StartTime/StopTime window (src/sim/mod.rs:1135-1150: E-type samples
        with start − dt ≤ t ≤ stop + dt, H-type start ≤ t ≤ stop + dt; stop
        ≤ 0: no limit); E-type series start with the initial state at t = 0,
        H-type ones end with the sample after the last step."""
        s = self.setup
        dt = s.dt
        v = self.series[p.name]
        width = v.shape[1] if v.ndim == 2 else 1
        if p.kind in PF.MAGNETIC or len(v):
            rows = PF.samples(p.kind, v, dt, 1)
        else:
            rows = [(0, 0.0, [0.0] * width)]  # a run of no steps: the initial state
        eps = 1e-9 * dt
        lo = p.start_time - (0.0 if p.kind in PF.MAGNETIC else dt) - eps
        return [r for r in rows if r[1] >= lo and (p.stop_time <= 0.0 or r[1] <= p.stop_time + dt + eps)]

    def files(self) -> dict:
        """File name → text of every probe file openEMS writes: the
        time-domain rows every ⌊N/OverSampling⌋ steps and, with
        FD_Samples, the frequency-domain file over the rows every N steps
        (N the Nyquist interval)."""
        s = self.setup
        dt = s.dt
        nyq = s.file.signal.nyquist_interval(dt)
        out = {}
        for p in s.probes:
            # The probe's own OverSampling, when set, replaces the <FDTD> one
            # (src/sim/results.rs:616-625).
            os_ = max(1, p.oversampling) if p.oversampling is not None else s.file.oversampling
            kt = max(1, nyq // os_)
            rows = self.rows(p)
            out[p.name] = PF.ProbeFile("time", p.kind, [[t] + list(x) for st, t, x in rows if st % kt == 0],
                                       p.location, PF.generator_text()).to_text()
            if p.fd:
                picked = [(t, np.asarray(x)) for st, t, x in rows if st % nyq == 0]
                w = 2.0 * nyq * dt
                fd_rows = []
                for f in p.fd:
                    acc = np.zeros(len(picked[0][1]) if picked else len(PF.COLUMNS[p.kind]), dtype=np.complex128)
                    for t, x in picked:
                        acc += w * np.exp(-2j * math.pi * f * t) * x
                    r = [float(f)]
                    for a in acc:
                        r += [a.real, a.imag]
                    fd_rows.append(r)
                out[p.name + "_FD"] = PF.ProbeFile("frequency", p.kind, fd_rows, p.location,
                                                   PF.generator_text()).to_text()
        return out

    def signal_files(self) -> dict:
        s = self.setup
        return {"et": s.file.signal.signal_text(s.dt, s.steps, 0.0),
                "ht": s.file.signal.signal_text(s.dt, s.steps, 0.5)}

    def write(self, directory: str) -> list:
        os.makedirs(directory, exist_ok=True)
        out = []
        for name, text in {**self.signal_files(), **self.files()}.items():  # a probe named et or ht wins
            path = os.path.join(directory, name)
            with open(path, "w") as h:
                h.write(text)
            out.append(path)
        return out


def load(path: str) -> Setup:
    with open(path) as h:
        return Setup(parse(h.read(), os.path.dirname(os.path.abspath(path))))


def loads(text: str) -> Setup:
    return Setup(parse(text))


def main(argv=None) -> int:
    """``python -m ems_b200.openems model.xml OUTDIR [--device N]``: runs an
    openEMS file on the CUDA engine and writes openEMS's probe files and
    ``et``/``ht`` into OUTDIR (the ems CLI's ``--openems`` output)."""
    import argparse

    from . import Engine

    ap = argparse.ArgumentParser(prog="python -m ems_b200.openems", description=main.__doc__)
    ap.add_argument("model")
    ap.add_argument("outdir")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    s = load(a.model)
    for w in s.warnings:
        print("warning:", w)
    eng = Engine(s.model, device=a.device)
    r = s.run(eng)
    paths = r.write(a.outdir)
    print(f"{len(paths)} files in {a.outdir}: {s.steps} steps of {s.dt:.6g} s")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
