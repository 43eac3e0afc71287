"""Test configuration: the ``gpu`` marker and shared helpers.

Tests marked ``gpu`` need a CUDA device (a B200); everything else runs on
the CPU: the oracle against the reference's known answers, the host-side
set-up, and that the C-ABI libraries load and export their symbols.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long CPU test")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the host library and the oracle once (the CUDA library too
    when nvcc is present, which it is here and on the GPU box)."""
    from ems_b200 import build as b
    from oracle import build as ob

    b.build_host()
    ob.build()
    try:
        b.build_gpu()
    except RuntimeError:
        pass
