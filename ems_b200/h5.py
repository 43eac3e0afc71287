"""HDF5 files for field dumps and probe series, in the layout of the
reference's ``src/io/h5.rs`` (``format`` = ``"ems-dump"`` or
``"ems-probes"``, ``version`` = 1), written from the HDF5 file format
specification with no HDF5 library.

Dump file (one per dump, ``write_time_dump`` / ``write_freq_dump``):

* root attributes ``format``, ``version`` (u32), ``name``, ``id`` (u32),
  ``quantity`` (``"E"``, ``"H"``, ``"J"``, ``"RotH"``, ``"D"``, ``"B"``),
  ``domain`` (``"time"`` / ``"frequency"``), ``position`` (``"nodes"``,
  ``"cell_centers"`` or ``"native"``), ``unit``; a frequency dump also
  ``samples`` (u64, the accumulated states);
* ``/mesh/x``, ``/mesh/y``, ``/mesh/z``: f64 sample coordinates, attribute
  ``unit = "m"``;
* time domain: ``/step`` (u64, completed steps of each snapshot), ``/time``
  (f64, attribute ``unit = "s"``); frequency domain: ``/frequency`` (f64,
  ``unit = "Hz"``);
* the field ``/<quantity>``, ``[n, nx, ny, nz, 3]`` in C order (z fastest,
  then the component): f32 in the time domain, the compound
  ``{r: f64, i: f64}`` (h5py's complex128) in the frequency domain, with its
  ``unit`` attribute.

Probe file (``write_probes``): root attributes ``format``, ``version``; one
group per probe (``group_name``, collisions suffixed ``_<id>``) with
attributes ``name``, ``kind``, ``id``, ``number``, ``dt`` and datasets
``time``, ``values`` (``[n]`` or ``[n, 3]``, with ``unit``) and, when the
probe has some, ``frequencies``.

Where this differs from the reference's files: the field dataset is stored
contiguously with a fixed shape, not in growable one-snapshot chunks (the
writer has every snapshot when it writes), and deflate is not offered. The
objects it writes are the specification's newer forms (superblock version
2, version 2 object headers with Jenkins lookup3 checksums, links held in
the group's header, contiguous or compact data, version 3 attribute
messages), which HDF5 1.8 and later read. ``read`` parses that subset back
(the tests read every file they write through it).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field
from typing import Any

import numpy as np

__all__ = ["lookup3", "group_name", "quantity_unit", "write_time_dump", "write_freq_dump", "write_probes",
           "time_dump_bytes", "freq_dump_bytes", "probes_bytes", "read", "LAYOUT_VERSION"]

LAYOUT_VERSION = 1
_UNDEF = 0xFFFFFFFFFFFFFFFF
_SIGNATURE = b"\x89HDF\r\n\x1a\n"
_M32 = 0xFFFFFFFF


# ---------------------------------------------------------------------------
# Jenkins lookup3 hashlittle (Bob Jenkins, 2006, public domain), the checksum
# the HDF5 format puts on superblocks and object headers (initial value 0).

def _rot(x: int, k: int) -> int:
    return ((x << k) | (x >> (32 - k))) & _M32


def lookup3(data: bytes, initval: int = 0) -> int:
    """``hashlittle(data, len(data), initval)``: the 32-bit lookup3 hash."""
    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & _M32
    if n == 0:
        return c
    pad = bytes(data) + b"\0" * ((12 - n % 12) % 12)
    blocks = len(pad) // 12
    for q in range(blocks):
        x, y, z = struct.unpack_from("<3I", pad, 12 * q)
        a, b, c = (a + x) & _M32, (b + y) & _M32, (c + z) & _M32
        if q == blocks - 1:
            break
        # mix(a, b, c)
        a = (a - c) & _M32; a ^= _rot(c, 4); c = (c + b) & _M32
        b = (b - a) & _M32; b ^= _rot(a, 6); a = (a + c) & _M32
        c = (c - b) & _M32; c ^= _rot(b, 8); b = (b + a) & _M32
        a = (a - c) & _M32; a ^= _rot(c, 16); c = (c + b) & _M32
        b = (b - a) & _M32; b ^= _rot(a, 19); a = (a + c) & _M32
        c = (c - b) & _M32; c ^= _rot(b, 4); b = (b + a) & _M32
    # final(a, b, c)
    c ^= b; c = (c - _rot(b, 14)) & _M32
    a ^= c; a = (a - _rot(c, 11)) & _M32
    b ^= a; b = (b - _rot(a, 25)) & _M32
    c ^= b; c = (c - _rot(b, 16)) & _M32
    a ^= c; a = (a - _rot(c, 4)) & _M32
    b ^= a; b = (b - _rot(a, 14)) & _M32
    c ^= b; c = (c - _rot(b, 24)) & _M32
    return c


# ---------------------------------------------------------------------------
# Datatypes (datatype message, class and version in the first byte).

@dataclass(frozen=True)
class _Type:
    kind: str            # "u32", "u64", "f32", "f64", "str", "c128"
    size: int

    def encode(self) -> bytes:
        if self.kind in ("u32", "u64"):  # fixed point, version 1, little endian, unsigned
            return bytes([0x10 | 0, 0, 0, 0]) + struct.pack("<I", self.size) + struct.pack("<HH", 0, 8 * self.size)
        if self.kind == "f32":  # IEEE single: implied mantissa msb, sign bit 31
            return (bytes([0x10 | 1, 0x20, 31, 0]) + struct.pack("<I", 4)
                    + struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127))
        if self.kind == "f64":
            return (bytes([0x10 | 1, 0x20, 63, 0]) + struct.pack("<I", 8)
                    + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023))
        if self.kind == "str":  # fixed length, null padded, ASCII
            return bytes([0x10 | 3, 0x01, 0, 0]) + struct.pack("<I", self.size)
        if self.kind == "c128":  # compound version 3: {r: f64 at 0, i: f64 at 8}
            f64 = _Type("f64", 8).encode()
            return (bytes([0x30 | 6, 2, 0, 0]) + struct.pack("<I", 16)
                    + b"r\0" + bytes([0]) + f64 + b"i\0" + bytes([8]) + f64)
        raise ValueError(self.kind)


_U32, _U64, _F32, _F64, _C128 = _Type("u32", 4), _Type("u64", 8), _Type("f32", 4), _Type("f64", 8), _Type("c128", 16)


def _dataspace(shape: tuple[int, ...] | None) -> bytes:
    """Dataspace message version 2: scalar (None) or simple."""
    if shape is None:
        return bytes([2, 0, 0, 0])
    return bytes([2, len(shape), 0, 1]) + b"".join(struct.pack("<Q", n) for n in shape)


def _pack(t: _Type, value: Any) -> bytes:
    if t.kind == "str":
        return value.encode("ascii")
    if t.kind == "u32":
        return struct.pack("<I", int(value))
    if t.kind == "u64":
        return struct.pack("<Q", int(value))
    if t.kind == "f64":
        return struct.pack("<d", float(value))
    if t.kind == "f32":
        return struct.pack("<f", float(value))
    raise ValueError(t.kind)


def _attr_value(v: Any) -> tuple[_Type, bytes]:
    if isinstance(v, str):
        if not v.isascii():
            raise ValueError(f"attribute string {v!r} is not ASCII")
        return _Type("str", max(1, len(v))), (v.encode("ascii") or b"\0")
    if isinstance(v, tuple) and len(v) == 2 and v[0] in ("u32", "u64", "f64"):
        t = {"u32": _U32, "u64": _U64, "f64": _F64}[v[0]]
        return t, _pack(t, v[1])
    if isinstance(v, float):
        return _F64, _pack(_F64, v)
    raise TypeError(f"attribute value {v!r}: use str, float or ('u32'|'u64'|'f64', value)")


def _attribute(name: str, value: Any) -> bytes:
    """Attribute message version 3 (scalar dataspace)."""
    t, data = _attr_value(value)
    nm = name.encode("ascii") + b"\0"
    dt, ds = t.encode(), _dataspace(None)
    return struct.pack("<BBHHHB", 3, 0, len(nm), len(dt), len(ds), 0) + nm + dt + ds + data


def _message(mtype: int, body: bytes, flags: int = 0) -> bytes:
    return struct.pack("<BHB", mtype, len(body), flags) + body


def _object_header(messages: list[bytes]) -> bytes:
    """Version 2 object header: "OHDR", version 2, flags (size of chunk 0 in
    four bytes), chunk 0 (the messages), lookup3 checksum."""
    body = b"".join(messages)
    head = b"OHDR" + bytes([2, 0x02]) + struct.pack("<I", len(body)) + body
    return head + struct.pack("<I", lookup3(head))


# ---------------------------------------------------------------------------
# The object tree and its serialisation.

@dataclass
class _Dataset:
    dtype: _Type
    shape: tuple[int, ...]
    data: bytes
    attrs: dict[str, Any] = field(default_factory=dict)


@dataclass
class _Group:
    attrs: dict[str, Any] = field(default_factory=dict)
    children: dict[str, Any] = field(default_factory=dict)

    def group(self, name: str) -> "_Group":
        g = _Group()
        self._add(name, g)
        return g

    def dataset(self, name: str, dtype: _Type, values, shape: tuple[int, ...] | None = None) -> _Dataset:
        a = np.ascontiguousarray(values)
        if dtype.kind == "c128":
            a = np.ascontiguousarray(np.asarray(values, dtype=np.complex128))
            raw = a.astype("<c16").tobytes()
        else:
            raw = a.astype({"u32": "<u4", "u64": "<u8", "f32": "<f4", "f64": "<f8"}[dtype.kind]).tobytes()
        d = _Dataset(dtype, tuple(int(n) for n in (a.shape if shape is None else shape)), raw)
        if int(np.prod(d.shape, dtype=np.int64)) * dtype.size != len(raw):
            raise ValueError(f"dataset {name!r}: {len(raw)} bytes for shape {d.shape}")
        self._add(name, d)
        return d

    def _add(self, name: str, obj) -> None:
        if not name or "/" in name or name in (".", ".."):
            raise ValueError(f"invalid object name {name!r}")
        if name in self.children:
            raise ValueError(f"duplicate object name {name!r}")
        name.encode("ascii")
        self.children[name] = obj


class _Writer:
    def __init__(self):
        self.buf = bytearray(48)  # the superblock, written last

    def _append(self, data: bytes, align: int = 8) -> int:
        self.buf += b"\0" * ((-len(self.buf)) % align)
        at = len(self.buf)
        self.buf += data
        return at

    def _place(self, obj) -> int:
        msgs = []
        if isinstance(obj, _Dataset):
            size = len(obj.data)
            if size <= 4096:  # compact: the raw data inside the layout message
                layout = struct.pack("<BBH", 3, 0, size) + obj.data
            else:
                addr = self._append(obj.data) if size else _UNDEF
                layout = struct.pack("<BBQQ", 3, 1, addr, size)
            msgs.append(_message(0x01, _dataspace(obj.shape)))
            msgs.append(_message(0x03, obj.dtype.encode(), flags=0x01))  # constant
            # Fill value version 3: allocated early, written if set, none defined.
            msgs.append(_message(0x05, bytes([3, 0x01 | (2 << 2)])))
            msgs.append(_message(0x08, layout))
        else:
            addrs = {name: self._place(child) for name, child in obj.children.items()}
            # Link info (compact storage: no heap, no index), group info.
            msgs.append(_message(0x02, struct.pack("<BBQQ", 0, 0, _UNDEF, _UNDEF)))
            msgs.append(_message(0x0A, bytes([0, 0])))
            for name, addr in addrs.items():
                nm = name.encode("ascii")
                if len(nm) > 255:
                    raise ValueError(f"object name {name!r} longer than 255 bytes")
                msgs.append(_message(0x06, bytes([1, 0, len(nm)]) + nm + struct.pack("<Q", addr)))
        for k, v in obj.attrs.items():
            msgs.append(_message(0x0C, _attribute(k, v)))
        return self._append(_object_header(msgs))

    def finish(self, root: _Group) -> bytes:
        root_addr = self._place(root)
        sb = _SIGNATURE + bytes([2, 8, 8, 0]) + struct.pack("<QQQQ", 0, _UNDEF, len(self.buf), root_addr)
        self.buf[:48] = sb + struct.pack("<I", lookup3(sb))
        return bytes(self.buf)


# ---------------------------------------------------------------------------
# The reference's files.

_QUANTITY_NAMES = ("E", "H", "J", "RotH", "D", "B")


def quantity_unit(quantity: str, freq: bool) -> str:
    """The ``unit`` attribute of a dump (src/io/h5.rs, ``quantity_unit``)."""
    base = {"E": ("V/m", "V*s/m"), "H": ("A/m", "A*s/m"), "J": ("A/m^2", "A*s/m^2"), "RotH": ("A/m^2", "A*s/m^2"),
            "D": ("C/m^2", "C*s/m^2"), "B": ("T", "T*s")}
    if quantity not in base:
        raise ValueError(f"unknown quantity {quantity!r}")
    return base[quantity][1 if freq else 0]


_POSITIONS = {0: "nodes", 1: "cell_centers", 2: "native", "nodes": "nodes", "cell_centers": "cell_centers",
              "native": "native"}


def _dump_root(name: str, id_: int, quantity: str, position, coords, freq: bool) -> _Group:
    if quantity not in _QUANTITY_NAMES:
        raise ValueError(f"unknown quantity {quantity!r}")
    root = _Group()
    root.attrs.update({"format": "ems-dump", "version": ("u32", LAYOUT_VERSION), "name": name, "id": ("u32", id_),
                       "quantity": quantity, "domain": "frequency" if freq else "time",
                       "position": _POSITIONS[position], "unit": quantity_unit(quantity, freq)})
    mesh = root.group("mesh")
    for axis, c in zip("xyz", coords):
        mesh.dataset(axis, _F64, np.asarray(c, np.float64)).attrs["unit"] = "m"
    return root


def _sampler_parts(sampler):
    """(quantity name, position, coords, dims) of an ems_b200.Sampler or a
    plain (quantity, position, (x, y, z)) tuple."""
    if isinstance(sampler, tuple):
        q, pos, coords = sampler
        dims = tuple(len(c) for c in coords)
        return q, pos, coords, dims
    coords = sampler.coords
    return sampler.name, sampler.position, coords, tuple(len(c) for c in coords)


def time_dump_bytes(name: str, id_: int, sampler, steps, times, values) -> bytes:
    """The bytes of a time-domain dump file (``h5::time_dump_bytes``):
    ``steps`` the completed steps of each snapshot, ``times`` their times
    [s], ``values`` (snapshots, nx, ny, nz, 3) or (snapshots, points, 3),
    stored as f32. ``sampler``: an ``ems_b200.Sampler`` or (quantity,
    position, (x, y, z))."""
    q, pos, coords, dims = _sampler_parts(sampler)
    steps = np.asarray(steps, np.uint64).reshape(-1)
    times = np.asarray(times, np.float64).reshape(-1)
    n = len(steps)
    if len(times) != n:
        raise ValueError("steps and times differ in length")
    v = np.asarray(values, np.float64)
    if v.size != n * int(np.prod(dims)) * 3:
        raise ValueError(f"values of {v.size} numbers for {n} snapshots of {dims} points")
    root = _dump_root(name, id_, q, pos, coords, False)
    root.dataset("step", _U64, steps)
    root.dataset("time", _F64, times).attrs["unit"] = "s"
    root.dataset(q, _F32, v.astype(np.float32), shape=(n, *dims, 3)).attrs["unit"] = quantity_unit(q, False)
    return _Writer().finish(root)


def freq_dump_bytes(name: str, id_: int, sampler, freqs, values, samples: int) -> bytes:
    """The bytes of a frequency-domain dump file (``h5::freq_dump_bytes``):
    ``values[k]`` the complex transform at ``freqs[k]``, (nx, ny, nz, 3) or
    (points, 3); ``samples`` the number of accumulated states."""
    q, pos, coords, dims = _sampler_parts(sampler)
    freqs = np.asarray(freqs, np.float64).reshape(-1)
    v = np.asarray(values, np.complex128)
    if v.size != len(freqs) * int(np.prod(dims)) * 3:
        raise ValueError(f"values of {v.size} numbers for {len(freqs)} frequencies of {dims} points")
    root = _dump_root(name, id_, q, pos, coords, True)
    root.attrs["samples"] = ("u64", int(samples))
    root.dataset("frequency", _F64, freqs).attrs["unit"] = "Hz"
    root.dataset(q, _C128, v, shape=(len(freqs), *dims, 3)).attrs["unit"] = quantity_unit(q, True)
    return _Writer().finish(root)


def group_name(name: str) -> str:
    """A probe's group name: ASCII letters, digits, ``-``, ``_`` and ``.``
    kept, everything else ``_``; ``_`` prefixed to "", "." and ".."."""
    s = "".join(c if (c.isascii() and c.isalnum()) or c in "-_." else "_" for c in name)
    return f"_{s}" if s in ("", ".", "..") else s


@dataclass
class ProbeSeries:
    """One probe's series for ``write_probes``: ``kind`` "voltage",
    "current", "efield" or "hfield"; ``values`` (n,) or (n, 3)."""
    name: str
    kind: str
    id: int
    number: int
    dt: float
    times: Any
    values: Any
    frequencies: Any = ()


_PROBE_UNITS = {"voltage": "V", "current": "A", "efield": "V/m", "hfield": "A/m"}


def probes_bytes(probes) -> bytes:
    """The bytes of a probe file (``h5::probes_bytes``)."""
    root = _Group()
    root.attrs.update({"format": "ems-probes", "version": ("u32", LAYOUT_VERSION)})
    used: set[str] = set()
    for p in probes:
        if p.kind not in _PROBE_UNITS:
            raise ValueError(f"probe {p.name!r}: unknown kind {p.kind!r}")
        g = group_name(p.name)
        if g in used:
            g = f"{g}_{p.id}"
            k = 2
            while g in used:
                g = f"{group_name(p.name)}_{p.id}_{k}"
                k += 1
        used.add(g)
        grp = root.group(g)
        grp.attrs.update({"name": p.name, "kind": p.kind, "id": ("u32", p.id), "number": ("u32", p.number),
                          "dt": ("f64", p.dt)})
        t = np.asarray(p.times, np.float64).reshape(-1)
        grp.dataset("time", _F64, t).attrs["unit"] = "s"
        v = np.asarray(p.values, np.float64)
        if v.shape not in ((len(t),), (len(t), 3)):
            raise ValueError(f"probe {p.name!r}: values of shape {v.shape} for {len(t)} times")
        grp.dataset("values", _F64, v).attrs["unit"] = _PROBE_UNITS[p.kind]
        fr = np.asarray(p.frequencies, np.float64).reshape(-1)
        if fr.size:
            grp.dataset("frequencies", _F64, fr)
    return _Writer().finish(root)


def _write(path: str, data: bytes) -> None:
    with open(path, "wb") as h:
        h.write(data)


def write_time_dump(path: str, name: str, id_: int, sampler, steps, times, values) -> None:
    """``h5::write_time_dump``: ``time_dump_bytes`` to ``path``."""
    _write(path, time_dump_bytes(name, id_, sampler, steps, times, values))


def write_freq_dump(path: str, name: str, id_: int, sampler, freqs, values, samples: int) -> None:
    """``h5::write_freq_dump``: ``freq_dump_bytes`` to ``path``."""
    _write(path, freq_dump_bytes(name, id_, sampler, freqs, values, samples))


def write_probes(path: str, probes) -> None:
    """``h5::write_probes``: ``probes_bytes`` to ``path``."""
    _write(path, probes_bytes(probes))


# ---------------------------------------------------------------------------
# Reader of the subset written above (superblock 2, version 2 object headers,
# compact links, contiguous or compact layouts, version 3 attributes).

class H5FormatError(ValueError):
    pass


def _parse_type(b: bytes, o: int) -> tuple[Any, int]:
    """(numpy dtype or "str", size) and the offset after the message."""
    cls, ver = b[o] & 0x0F, b[o] >> 4
    bits = b[o + 1] | (b[o + 2] << 8) | (b[o + 3] << 16)
    size = struct.unpack_from("<I", b, o + 4)[0]
    p = o + 8
    if cls == 0:
        signed = bool(bits & 0x08)
        if bits & 0x01:
            raise H5FormatError("big-endian integers")
        return np.dtype(f"<{'i' if signed else 'u'}{size}"), p + 4
    if cls == 1:
        if bits & 0x01:
            raise H5FormatError("big-endian floats")
        return np.dtype(f"<f{size}"), p + 12
    if cls == 3:
        return ("str", size), p
    if cls == 6:
        if ver != 3:
            raise H5FormatError(f"compound datatype version {ver}")
        n = bits & 0xFFFF
        names, offs = [], []
        width = max(1, (size.bit_length() + 7) // 8)
        members = []
        for _ in range(n):
            e = b.index(b"\0", p)
            nm = b[p:e].decode()
            p = e + 1
            off = int.from_bytes(b[p:p + width], "little")
            p += width
            t, p = _parse_type(b, p)
            members.append((nm, off, t))
            names.append(nm)
            offs.append(off)
        if [m[0] for m in members] == ["r", "i"] and all(m[2] == np.dtype("<f8") for m in members) and size == 16:
            return np.dtype("<c16"), p
        return np.dtype({"names": names, "formats": [m[2] for m in members], "offsets": offs, "itemsize": size}), p
    raise H5FormatError(f"datatype class {cls}")


def _parse_space(b: bytes, o: int) -> tuple[int, ...] | None:
    ver, rank, flags, typ = b[o], b[o + 1], b[o + 2], b[o + 3]
    if ver != 2:
        raise H5FormatError(f"dataspace version {ver}")
    if typ == 0:
        return None
    return tuple(struct.unpack_from(f"<{rank}Q", b, o + 4)) if rank else ()


def _decode(raw: bytes, t, shape):
    if isinstance(t, tuple):  # fixed-length string
        s = raw[:t[1]].split(b"\0", 1)[0].decode("ascii")
        return s
    a = np.frombuffer(raw, dtype=t)
    return a[0] if shape is None else a.reshape(shape)


def _parse_header(b: bytes, addr: int) -> list[tuple[int, bytes]]:
    if b[addr:addr + 4] != b"OHDR" or b[addr + 4] != 2:
        raise H5FormatError(f"no version 2 object header at {addr}")
    flags = b[addr + 5]
    p = addr + 6
    if flags & 0x20:
        p += 16
    if flags & 0x10:
        p += 4
    width = 1 << (flags & 0x03)
    size = int.from_bytes(b[p:p + width], "little")
    p += width
    end = p + size
    if struct.unpack_from("<I", b, end)[0] != lookup3(b[addr:end]):
        raise H5FormatError(f"object header checksum at {addr}")
    out = []
    while p + 4 <= end:
        mtype, msize, mflags = struct.unpack_from("<BHB", b, p)
        p += 4
        if flags & 0x04:
            p += 2
        out.append((mtype, b[p:p + msize]))
        p += msize
    return out


def _parse_attribute(m: bytes) -> tuple[str, Any]:
    ver, _, nsz, tsz, ssz, _ = struct.unpack_from("<BBHHHB", m, 0)
    if ver != 3:
        raise H5FormatError(f"attribute version {ver}")
    p = 9
    name = m[p:p + nsz].split(b"\0", 1)[0].decode()
    p += nsz
    t, _ = _parse_type(m, p)
    p += tsz
    shape = _parse_space(m, p)
    p += ssz
    return name, _decode(m[p:], t, shape)


def _read_object(b: bytes, addr: int) -> dict:
    msgs = _parse_header(b, addr)
    attrs, links = {}, {}
    space = dtype = layout = None
    for mtype, m in msgs:
        if mtype == 0x0C:
            k, v = _parse_attribute(m)
            attrs[k] = v
        elif mtype == 0x06:
            ver, fl = m[0], m[1]
            if ver != 1 or fl & 0x08:
                raise H5FormatError("only hard links")
            p = 2 + (8 if fl & 0x04 else 0) + (1 if fl & 0x10 else 0)
            w = 1 << (fl & 0x03)
            ln = int.from_bytes(m[p:p + w], "little")
            p += w
            name = m[p:p + ln].decode()
            links[name] = struct.unpack_from("<Q", m, p + ln)[0]
        elif mtype == 0x01:
            space = _parse_space(m, 0)
        elif mtype == 0x03:
            dtype, _ = _parse_type(m, 0)
        elif mtype == 0x08:
            layout = m
    out: dict = {"attrs": attrs}
    if layout is not None:
        if layout[0] != 3:
            raise H5FormatError(f"layout version {layout[0]}")
        if layout[1] == 0:
            n = struct.unpack_from("<H", layout, 2)[0]
            raw = layout[4:4 + n]
        elif layout[1] == 1:
            addr_d, n = struct.unpack_from("<QQ", layout, 2)
            raw = b"" if addr_d == _UNDEF else b[addr_d:addr_d + n]
        else:
            raise H5FormatError("chunked layout")
        out["data"] = _decode(raw, dtype, space if space is not None else None)
    for name, a in links.items():
        out[name] = _read_object(b, a)
    return out


def read(source) -> dict:
    """A file written by this module (path or bytes) as nested dicts: each
    object {"attrs": {...}, <child name>: {...}, ...}, datasets with "data"
    (numpy; the complex compound as complex128, strings as str)."""
    b = source if isinstance(source, (bytes, bytearray)) else open(source, "rb").read()
    b = bytes(b)
    if b[:8] != _SIGNATURE or b[8] != 2:
        raise H5FormatError("not an HDF5 file with a version 2 superblock")
    if struct.unpack_from("<I", b, 44)[0] != lookup3(b[:44]):
        raise H5FormatError("superblock checksum")
    eof, root = struct.unpack_from("<QQ", b, 28)
    if eof != len(b):
        raise H5FormatError(f"end-of-file address {eof} for {len(b)} bytes")
    return _read_object(b, root)
