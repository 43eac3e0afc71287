"""VTK XML ``RectilinearGrid`` (``.vtr``) and ``.pvd`` collection writers for
field dumps (src/io/vtr.rs; the dump side, src/engine/dump.rs:977-983,
1143-1192, 1250-1258, 1560-1586).

The file layout is Kitware's XML format: one ``<RectilinearGrid>`` with one
``<Piece>``, whose ``<PointData>``, ``<CellData>`` and ``<Coordinates>`` hold
``<DataArray>`` elements; ``TimeValue`` and other dataset-wide values go to
``<FieldData>``. Tuples are written x fastest; inputs are z fastest (the
engine's order, ``layout="z"``) or already x fastest (``layout="x"``).
Encodings: inline base64 ``binary`` (default; a little-endian byte-count
header, UInt64 by default, then the values, encoded as one stream),
``ascii`` (shortest round-trip decimal in exponent notation, six per line)
or raw ``appended`` data. A complex array becomes ``name_re``/``name_im``
(or ``name_mag``/``name_phase``). The output is the reference's byte for
byte for the same inputs.
"""
from __future__ import annotations

import base64
import math
import os
import struct
from dataclasses import dataclass
from typing import Sequence

import numpy as np

__all__ = ["VtrWriter", "PvdCollection", "rust_exp", "write_time_dump", "write_freq_dump", "snapshot_file"]

_PER_LINE = 6


def rust_exp(v, single: bool = False) -> str:
    """A float in exponent notation with the fewest digits that read back
    to the same value (``format!("{:e}")`` of f64, or of f32 when ``single``):
    ``1e0``, ``-2.5e-3``, ``NaN``, ``inf``."""
    x = float(v)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    if x == 0.0:
        return "-0e0" if math.copysign(1.0, x) < 0 else "0e0"
    s = np.format_float_scientific(np.float32(x) if single else np.float64(x), unique=True, trim="-")
    mant, exp = s.split("e")
    return f"{mant}e{int(exp)}"


def escape(s: str) -> str:
    """An attribute value inside double quotes (src/io/vtr.rs:930-947)."""
    out = []
    for ch in s:
        out.append({"&": "&amp;", "<": "&lt;", ">": "&gt;", '"': "&quot;", "'": "&apos;", "\n": "&#10;",
                    "\r": "&#13;", "\t": "&#9;"}.get(ch, ch))
    return "".join(out)


@dataclass
class _Entry:
    name: str
    cell: bool
    values: np.ndarray  # (tuples, ncomp) in x-fastest order, f32 or f64

    @property
    def ncomp(self) -> int:
        return self.values.shape[1]


class VtrWriter:
    """One ``.vtr`` file on the rectilinear grid ``x``, ``y``, ``z`` (metres,
    each non-empty and strictly increasing); ``encoding`` "binary", "ascii"
    or "appended", ``header`` "UInt64" or "UInt32"."""

    def __init__(self, x: Sequence[float], y: Sequence[float], z: Sequence[float], encoding: str = "binary",
                 header: str = "UInt64"):
        if encoding not in ("binary", "ascii", "appended") or header not in ("UInt64", "UInt32"):
            raise ValueError("VTK: unknown encoding or header type")
        self.coords = [np.asarray(c, dtype=np.float64) for c in (x, y, z)]
        self.encoding, self.header = encoding, header
        self.time: float | None = None
        self.fields: list = []
        self.entries: list = []
        self._pending: list = []

    # ---- building
    def set_time(self, t: float) -> "VtrWriter":
        self.time = float(t)
        return self

    def field(self, name: str, values: Sequence[float]) -> "VtrWriter":
        self.fields.append((name, np.asarray(values, dtype=np.float64).ravel()))
        return self

    def point(self, name: str, data, layout: str = "z") -> "VtrWriter":
        self._pending.append((name, False, data, layout))
        return self

    def cell(self, name: str, data, layout: str = "z") -> "VtrWriter":
        self._pending.append((name, True, data, layout))
        return self

    def point_complex(self, name: str, re, im, layout: str = "z", form: str = "reim") -> "VtrWriter":
        return self._complex(name, False, re, im, layout, form)

    def cell_complex(self, name: str, re, im, layout: str = "z", form: str = "reim") -> "VtrWriter":
        return self._complex(name, True, re, im, layout, form)

    def _complex(self, name, cell, re, im, layout, form):
        re, im = np.asarray(re), np.asarray(im)
        if re.shape != im.shape:
            raise ValueError(f"VTK array {name!r}: real and imaginary parts have different shapes")
        if form == "reim":
            parts = [("_re", re), ("_im", im)]
        else:
            parts = [("_mag", np.hypot(re, im).astype(re.dtype)), ("_phase", np.arctan2(im, re).astype(re.dtype))]
        for suffix, v in parts:
            self._pending.append((name + suffix, cell, v, layout))
        return self

    # ---- geometry
    def point_dims(self):
        return [len(c) for c in self.coords]

    def cell_dims(self):
        return [max(len(c) - 1, 1) for c in self.coords]

    def _validate(self):
        for name, c in zip("xyz", self.coords):
            if c.size == 0:
                raise ValueError(f"VTK grid: no {name} coordinates")
            if not np.all(np.isfinite(c)):
                raise ValueError(f"VTK grid: non-finite {name} coordinate")
            if np.any(np.diff(c) <= 0):
                raise ValueError(f"VTK grid: {name} coordinates are not strictly increasing")
        entries = []
        for name, cell, data, layout in self._pending:
            dims = self.cell_dims() if cell else self.point_dims()
            n = int(np.prod(dims))
            a = np.asarray(data)
            if a.dtype not in (np.float32, np.float64):
                a = a.astype(np.float64)
            if a.ndim == 1:
                a = a[:, None]
            else:
                a = a.reshape(-1, a.shape[-1])
            if a.shape[1] not in (1, 3):
                raise ValueError(f"VTK array {name!r}: scalars or 3-vectors only")
            if a.shape[0] != n:
                raise ValueError(f"VTK array {name!r}: {a.shape[0]} tuples given, the grid needs {n}")
            if not name:
                raise ValueError("VTK array with an empty name")
            if any(e.cell == cell and e.name == name for e in entries):
                raise ValueError(f"duplicate VTK array name {name!r}")
            if layout == "z":  # (i·dy + j)·dz + k → x fastest
                a = a.reshape(dims[0], dims[1], dims[2], -1).transpose(2, 1, 0, 3).reshape(n, -1)
            if self.encoding != "ascii" and self.header == "UInt32" and a.nbytes > 0xFFFFFFFF:
                raise ValueError(f"array of {a.nbytes} bytes needs a UInt64 header")
            entries.append(_Entry(name, cell, np.ascontiguousarray(a)))
        names = []
        for name, _ in self.fields:
            if not name:
                raise ValueError("VTK field data with an empty name")
            if name in names or (self.time is not None and name == "TimeValue"):
                raise ValueError(f"duplicate VTK field data name {name!r}")
            names.append(name)
        self.entries = entries

    # ---- output
    def _hdr(self, nbytes: int) -> bytes:
        return struct.pack("<Q" if self.header == "UInt64" else "<I", nbytes)

    def _ascii(self, values: np.ndarray, single: bool) -> str:
        flat = values.ravel()
        lines = []
        for q in range(0, flat.size, _PER_LINE):
            lines.append("          " + " ".join(rust_exp(v, single) for v in flat[q:q + _PER_LINE]) + "\n")
        return "".join(lines)

    def _inline(self, values: np.ndarray) -> str:
        raw = values.astype(values.dtype.newbyteorder("<"), copy=False).tobytes()
        if self.encoding == "ascii":
            return self._ascii(values, values.dtype == np.float32)
        return "          " + base64.b64encode(self._hdr(len(raw)) + raw).decode("ascii") + "\n"

    def to_bytes(self) -> bytes:
        self._validate()
        pd = self.point_dims()
        ext = f"0 {pd[0] - 1} 0 {pd[1] - 1} 0 {pd[2] - 1}"
        out = ['<?xml version="1.0"?>\n',
               f'<VTKFile type="RectilinearGrid" version="1.0" byte_order="LittleEndian" header_type="{self.header}">\n',
               f'  <RectilinearGrid WholeExtent="{ext}">\n']
        fd = ([("TimeValue", np.array([self.time]))] if self.time is not None else []) + list(self.fields)
        if fd:
            out.append("    <FieldData>\n")
            for name, v in fd:
                out.append(f'      <DataArray type="Float64" Name="{escape(name)}" NumberOfTuples="{len(v)}" '
                           f'format="ascii">\n')
                out.append(self._ascii(v, False))
                out.append("      </DataArray>\n")
            out.append("    </FieldData>\n")
        out.append(f'    <Piece Extent="{ext}">\n')
        offset = 0
        appended = []
        hsize = 8 if self.header == "UInt64" else 4

        def open_array(tname, name, ncomp, nbytes):
            nonlocal offset
            head = f'        <DataArray type="{tname}" Name="{escape(name)}" NumberOfComponents="{ncomp}"'
            if self.encoding == "ascii":
                return head + ' format="ascii">\n'
            if self.encoding == "binary":
                return head + ' format="binary">\n'
            s = head + f' format="appended" offset="{offset}">'
            offset += hsize + nbytes
            return s

        close = "</DataArray>\n" if self.encoding == "appended" else "        </DataArray>\n"
        for cell, tag in ((False, "PointData"), (True, "CellData")):
            es = [e for e in self.entries if e.cell == cell]
            if not es:
                continue
            head = f"      <{tag}"
            for attr, nc in (("Scalars", 1), ("Vectors", 3)):
                first = next((e for e in es if e.ncomp == nc), None)
                if first is not None:
                    head += f' {attr}="{escape(first.name)}"'
            out.append(head + ">\n")
            for e in es:
                tname = "Float32" if e.values.dtype == np.float32 else "Float64"
                out.append(open_array(tname, e.name, e.ncomp, e.values.nbytes))
                if self.encoding == "appended":
                    appended.append(e.values)
                else:
                    out.append(self._inline(e.values))
                out.append(close)
            out.append(f"      </{tag}>\n")
        out.append("      <Coordinates>\n")
        for name, c in zip("xyz", self.coords):
            out.append(open_array("Float64", name, 1, c.nbytes))
            if self.encoding == "appended":
                appended.append(c)
            else:
                out.append(self._inline(c))
            out.append(close)
        out.append("      </Coordinates>\n    </Piece>\n  </RectilinearGrid>\n")
        data = "".join(out).encode("utf-8")
        if self.encoding == "appended":
            blob = b"".join(self._hdr(a.nbytes) + a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes()
                            for a in appended)
            data += b'  <AppendedData encoding="raw">\n   _' + blob + b"\n  </AppendedData>\n"
        return data + b"</VTKFile>\n"

    def write(self, path: str) -> None:
        data = self.to_bytes()
        with open(path, "wb") as h:
            h.write(data)


class PvdCollection:
    """A ParaView ``.pvd`` list of datasets with their time step (or
    frequency) (src/io/vtr.rs:960-1075)."""

    def __init__(self):
        self.entries: list[tuple[float, int, str]] = []

    def push(self, timestep: float, file: str, part: int = 0) -> "PvdCollection":
        self.entries.append((float(timestep), int(part), file))
        return self

    def to_bytes(self) -> bytes:
        for t, _, f in self.entries:
            if not math.isfinite(t):
                raise ValueError(f"pvd: non-finite time step for {f!r}")
            if not f:
                raise ValueError("pvd: empty file name")
        out = ['<?xml version="1.0"?>\n', '<VTKFile type="Collection" version="0.1" byte_order="LittleEndian">\n',
               "  <Collection>\n"]
        for t, p, f in self.entries:
            out.append(f'    <DataSet timestep="{rust_exp(t)}" group="" part="{p}" file="{escape(f)}"/>\n')
        out.append("  </Collection>\n</VTKFile>\n")
        return "".join(out).encode("utf-8")

    def write(self, path: str) -> None:
        data = self.to_bytes()
        with open(path, "wb") as h:
            h.write(data)


def snapshot_file(basename: str, step: int) -> str:
    """``<basename>_<step>.vtr`` with the step zero-padded to 8 digits (dump.rs:1139-1141)."""
    return f"{basename}_{step:08d}.vtr"


def write_time_dump(sampler, states, values, dt: float, directory: str, basename: str) -> None:
    """``TimeDump::write_vtr`` (dump.rs:1250-1258, 1182-1192): one file per
    snapshot, point vectors named after the quantity in f32 (the reference's
    snapshots hold f32), ``TimeValue`` the quantity's time, and the ``.pvd``
    index. ``values``: (snapshots, points, 3) or (snapshots, dx, dy, dz, 3)."""
    os.makedirs(directory, exist_ok=True)
    pvd = PvdCollection()
    for m, v in zip(states, values):
        t = sampler.time(int(m), dt)
        f = snapshot_file(basename, int(m))
        VtrWriter(*sampler.coords).set_time(t).point(sampler.name, np.asarray(v, np.float64).reshape(-1, 3)
                                                     .astype(np.float32)).write(os.path.join(directory, f))
        pvd.push(t, f)
        pvd.write(os.path.join(directory, f"{basename}.pvd"))


def write_freq_dump(sampler, freqs, values, directory: str, basename: str) -> None:
    """``FreqDump::write_vtr`` (dump.rs:1560-1586): one ``<basename>_f<k>.vtr``
    per frequency with ``<Q>_re``/``<Q>_im`` point vectors (f64), ``TimeValue``
    and a ``Frequency`` entry of that frequency, and the ``.pvd`` indexed by
    frequency. ``values[k]``: complex (points, 3) or (dx, dy, dz, 3)."""
    os.makedirs(directory, exist_ok=True)
    pvd = PvdCollection()
    for k, f in enumerate(freqs):
        v = np.asarray(values[k]).reshape(-1, 3)
        name = f"{basename}_f{k}.vtr"
        (VtrWriter(*sampler.coords).set_time(f).field("Frequency", [f])
         .point_complex(sampler.name, v.real.astype(np.float64), v.imag.astype(np.float64))
         .write(os.path.join(directory, name)))
        pvd.push(f, name)
    pvd.write(os.path.join(directory, f"{basename}.pvd"))
