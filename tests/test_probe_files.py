"""openEMS probe text files (ems_b200/probe_files.py) against the files in
the reference's openEMS fixtures (tests/fixtures/openems/*: openEMS v0.37
output): every fixture probe file parses, and written back from its parsed
numbers reproduces every line byte for byte but the generator line. Plus
the sampling rules on engine series: the E-type initial row, H-type half
steps, the file interval and the factor-2 frequency-domain sum. CPU only;
the fixture tests skip when the reference tree is not present."""
import glob
import math
import os

import numpy as np
import pytest

from ems_b200 import probe_files as PF

# The reference tree's openEMS fixtures; EMS_REFERENCE_FIXTURES overrides the location.
FIXTURES = os.environ.get("EMS_REFERENCE_FIXTURES", "/root/reference/tests/fixtures/openems")


def _probe_files():
    out = []
    for d in sorted(glob.glob(os.path.join(FIXTURES, "*"))):
        for f in sorted(glob.glob(os.path.join(d, "*"))):
            base = os.path.basename(f)
            if base.endswith((".txt", ".xml")) or not os.path.isfile(f):
                continue
            with open(f, errors="replace") as h:
                first = h.readline()
            if first.startswith("% time-domain") or first.startswith("% frequency-domain"):
                if any(t in first for t in PF.TITLES.values()):
                    out.append(f)
    return out


@pytest.mark.skipif(not os.path.isdir(FIXTURES), reason="reference fixtures not present")
def test_fixture_probe_files_round_trip_byte_for_byte():
    files = _probe_files()
    assert len(files) > 50
    for f in files:
        text = open(f).read()
        p = PF.parse(text)
        got = p.to_text().splitlines()
        want = text.splitlines()
        assert len(got) == len(want), f
        assert got[1:] == want[1:], (f, next(((a, b) for a, b in zip(got[1:], want[1:]) if a != b), None))


def test_format_g_is_c_printf():
    assert PF.fmt_g(1.92583319e-12, 6) == "1.92583e-12"
    assert PF.fmt_g(2.5e9, 6) == "2.5e+09"
    assert PF.fmt_g(0.012, 6) == "0.012"
    assert PF.fmt_g(-0.0, 12) == "-0" and PF.fmt_g(0.0, 12) == "0"
    assert PF.fmt_g(4.04424970893e-11, 12) == "4.04424970893e-11"
    assert PF.fmt_g(float("nan"), 6) == "nan"


def test_sampling_rules_of_engine_series():
    dt = 2e-12
    v = np.arange(1, 7, dtype=float)  # voltage after steps 0..5
    td = PF.time_domain("voltage", v, dt)
    assert td.rows[0] == [0.0, 0.0]                       # the initial state
    assert td.rows[1][0] == pytest.approx(dt) and td.rows[1][1] == 1.0
    i = np.arange(1, 7, dtype=float)
    tdi = PF.time_domain("current", i, dt)
    assert tdi.rows[0][0] == pytest.approx(0.5 * dt) and len(tdi.rows) == 6
    td2 = PF.time_domain("voltage", v, dt, file_interval=2)
    assert [r[0] / dt for r in td2.rows] == pytest.approx([0, 2, 4, 6])
    fd = PF.frequency_domain("voltage", v, dt, [1e9], nyquist=2)
    t = np.array([0, 2, 4, 6]) * dt
    x = np.array([0.0, 2.0, 4.0, 6.0])
    want = 2.0 * 2 * dt * np.sum(x * np.exp(-2j * math.pi * 1e9 * t))
    assert fd.rows[0][1] == pytest.approx(want.real) and fd.rows[0][2] == pytest.approx(want.imag)
    text = fd.to_text()
    assert text.splitlines()[1] == "% f/Hz\tvoltage\t" and text.splitlines()[2] == "%\treal\timag"
