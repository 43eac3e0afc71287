"""openEMS probe text files: writer and reader for the engine's series.

Restates the reference's io/openems/probes.rs (src/io/openems/probes.rs:
1-76 format, 340-398 to_text, 399-460 time/frequency domain, 465-492
sample assembly, 557-598 number format) so a run of this engine can hand
the ems CLI's tools the same files:

    % time-domain voltage integration by <program> @<date>
    % start-coordinates: (x,y,z) m -> [i,j,k]
    % stop-coordinates: (x,y,z) m -> [i,j,k]
    % t/s\tvoltage
    0\t0
    4.04424970893e-11\t-8.83796715812e-08

Columns are tab-separated; time-domain values are printed like C's
``%.12g``, frequency-domain values and coordinates like ``%g``. E-type
files (voltage, E field) carry the initial state as a row at t = 0 when the
series starts at the first step; H-type rows sit at (k + ½)·dt. The
frequency-domain value at f is X(f) = 2·Σ_k x(t_k)·e^{−j2πf·t_k}·K·dt over
the samples every K steps (K the Nyquist interval), the convention the
reference established against openEMS.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

TITLES = {
    "voltage": "voltage integration",
    "current": "current integration",
    "efield": "electric field probe",
    "hfield": "magnetic field probe",
    "voltage_mode": "voltage mode matching",
    "current_mode": "current mode matching",
}
COLUMNS = {
    "voltage": ["voltage"],
    "current": ["current"],
    "efield": ["Ex/(V/m)", "Ey/(V/m)", "Ez/(V/m)"],
    "hfield": ["Hx/(A/m)", "Hy/(A/m)", "Hz/(A/m)"],
    "voltage_mode": ["voltage", "mode_purity"],
    "current_mode": ["current", "mode_purity"],
}
MAGNETIC = {"current", "hfield", "current_mode"}


def fmt_g(v: float, prec: int) -> str:
    """C ``printf("%.{prec}g")`` (src/io/openems/probes.rs:572-598)."""
    v = float(v)
    if v == 0.0:
        return "-0" if math.copysign(1.0, v) < 0 else "0"
    if math.isnan(v):
        return "nan"
    if math.isinf(v):
        return "-inf" if v < 0 else "inf"
    return "%.*g" % (max(1, prec), v)


@dataclass
class ProbeFile:
    """One openEMS probe file: domain "time" or "frequency", kind (voltage,
    current, efield, hfield), location ((start coords m, start index),
    (stop coords m, stop index)) or None, and rows (abscissa then values;
    frequency rows: real and imaginary part per component)."""

    domain: str
    kind: str
    rows: list = field(default_factory=list)
    location: tuple | None = None
    generator: str = ""

    def to_text(self) -> str:
        dom = "time-domain" if self.domain == "time" else "frequency-domain"
        out = [f"% {dom} {TITLES[self.kind]} by {self.generator}"]
        if self.location is not None:
            for what, (c, i) in zip(("start", "stop"), self.location):
                out.append(f"% {what}-coordinates: ({fmt_g(c[0], 6)},{fmt_g(c[1], 6)},{fmt_g(c[2], 6)}) m -> "
                           f"[{i[0]},{i[1]},{i[2]}]")
        prec, absc = (12, "t/s") if self.domain == "time" else (6, "f/Hz")
        head = "% " + absc
        for c in COLUMNS[self.kind]:
            head += "\t" + c + ("\t" if self.domain == "frequency" else "")
        out.append(head)
        if self.domain == "frequency":
            out.append("%" + "\treal\timag" * len(COLUMNS[self.kind]))
        for r in self.rows:
            out.append("\t".join(fmt_g(v, prec) for v in r))
        return "\n".join(out) + "\n"

    def write(self, path: str) -> None:
        with open(path, "w") as f:
            f.write(self.to_text())


def parse(text: str) -> ProbeFile:
    """Reads an openEMS probe file (src/io/openems/probes.rs ProbeFile::parse)."""
    lines = text.splitlines()
    if not lines or not lines[0].startswith("%"):
        raise ValueError("not an openEMS probe file")
    head = lines[0].lstrip("%").strip()
    if head.startswith("time-domain"):
        domain = "time"
    elif head.startswith("frequency-domain"):
        domain = "frequency"
    else:
        raise ValueError(f"unknown domain in {lines[0]!r}")
    kind = next((k for k, t in TITLES.items() if f" {t} " in f" {head} "), None)
    if kind is None:
        raise ValueError(f"unknown probe kind in {lines[0]!r}")
    generator = head.split(" by ", 1)[1] if " by " in head else ""
    loc, rows = [], []
    for ln in lines[1:]:
        if ln.startswith("%"):
            c = ln.lstrip("%").strip()
            if c.startswith(("start-coordinates:", "stop-coordinates:")):
                xyz = [float(x) for x in c[c.index("(") + 1:c.index(")")].split(",")]
                ijk = [int(x) for x in c[c.index("[") + 1:c.index("]")].split(",")]
                loc.append((xyz, ijk))
            continue
        if ln.strip():
            rows.append([float(x) for x in ln.split("\t")])
    return ProbeFile(domain, kind, rows, tuple(loc) if len(loc) == 2 else None, generator)


def generator_text() -> str:
    return "ems_b200 @" + time.asctime(time.gmtime())


def samples(kind: str, series: np.ndarray, dt: float, interval: int = 1):
    """(step, time, value) rows of an engine series (a probe sampled at
    every `interval` steps from step 0: voltage after the E update of step
    n at (n+1)·dt, current after the H update at (n+½)·dt), with the E-type
    initial state as a row at t = 0 when the samples start at the first
    step (src/io/openems/probes.rs:465-492)."""
    series = np.asarray(series, dtype=np.float64).reshape(len(series), -1)
    mag = kind in MAGNETIC
    out = []
    n = np.arange(len(series)) * interval
    t = (n + 0.5) * dt if mag else (n + 1.0) * dt
    step = np.maximum(0, np.round(t / dt - (0.5 if mag else 0.0))).astype(np.int64)
    if not mag and len(step) and step[0] == 1:
        out.append((0, 0.0, [0.0] * series.shape[1]))
    out.extend((int(s), float(tt), list(v)) for s, tt, v in zip(step, t, series))
    return out


def time_domain(kind: str, series, dt: float, interval: int = 1, file_interval: int = 1, location=None):
    """The time-domain file: the rows whose step is a multiple of
    `file_interval` (src/io/openems/probes.rs:399-419)."""
    rows = [[t] + v for s, t, v in samples(kind, series, dt, interval) if s % max(1, file_interval) == 0]
    return ProbeFile("time", kind, rows, location, generator_text())


def frequency_domain(kind: str, series, dt: float, freqs, nyquist: int, interval: int = 1, location=None):
    """The frequency-domain file: X(f) = 2·Σ_k x(t_k)·e^{−j2πf·t_k}·K·dt over
    the samples every K = nyquist steps (src/io/openems/probes.rs:425-460)."""
    n = max(1, nyquist)
    picked = [(t, v) for s, t, v in samples(kind, series, dt, interval) if s % n == 0]
    w = 2.0 * n * dt
    rows = []
    for f in freqs:
        acc = np.zeros(len(picked[0][1]) if picked else len(COLUMNS[kind]), dtype=np.complex128)
        for t, v in picked:
            acc += w * np.exp(-2j * math.pi * f * t) * np.asarray(v)
        r = [float(f)]
        for a in acc:
            r += [a.real, a.imag]
        rows.append(r)
    return ProbeFile("frequency", kind, rows, location, generator_text())
