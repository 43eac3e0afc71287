"""The oracle: a CPU restatement of the reference engine's step.

TEST INFRASTRUCTURE ONLY — the checker the CUDA engine is compared with in
tests/, in ``__graft_entry__.smoke()`` and as ``bench.py``'s CPU baseline.
Nothing in ``ems_b200`` imports it. :class:`OracleEngine` consumes the same
engine descriptor (include/ems_gpu.h) as ``ems_b200.Engine`` and has the
same interface.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = C.CDLL(_build.build())
        p = C.c_void_p
        for name, args in {
            "oracle_create": [p, C.c_int, p],
            "oracle_destroy": [p],
            "oracle_threads": [p],
            "oracle_set_curl_order": [p, C.c_int],
            "oracle_upml_state": [p, C.c_size_t, C.c_int, p, p, C.c_size_t],
            "oracle_run": [p, C.c_uint64],
            "oracle_step_with_energy": [p, p],
            "oracle_download_field": [p, C.c_int, C.c_int, p],
            "oracle_upload_field": [p, C.c_int, C.c_int, p],
            "oracle_samples": [p, C.c_size_t, C.c_int, p, C.c_size_t, p],
            "oracle_sample": [p, p, p],
        }.items():
            f = getattr(L, name)
            f.restype = C.c_int
            f.argtypes = args
        _lib = L
    return _lib


class OracleEngine:
    """CPU engine for a built ``ems_b200.Model`` (threads=0: the reference's default rule)."""

    def __init__(self, model, threads: int = 0):
        self._lib = lib()
        self._model = model
        h = C.c_void_p()
        st = self._lib.oracle_create(model.desc, threads, C.byref(h))
        if st != 0:
            raise RuntimeError(f"oracle_create failed ({st})")
        self._h = h
        self.nodes = model.nodes
        self.dt = model.dt

    @property
    def threads(self) -> int:
        return self._lib.oracle_threads(self._h)

    def upml_state(self, op: int, side: int, n: int):
        """(F, v) of the openEMS PML operator ``op``, side 0 E / 1 H."""
        f = np.empty(n, dtype=np.float32)
        v = np.empty(n, dtype=np.float32)
        if n and self._lib.oracle_upml_state(self._h, op, side, f.ctypes.data, v.ctypes.data, n) != 0:
            raise ValueError("not a PML operator")
        return f, v

    def set_curl_order(self, order: int) -> None:
        """0 the reference's default summation order, 1 openEMS's."""
        if self._lib.oracle_set_curl_order(self._h, order) != 0:
            raise ValueError(f"invalid curl order {order}")

    def run(self, n: int) -> None:
        if self._lib.oracle_run(self._h, n) != 0:
            raise RuntimeError("oracle_run failed")

    def step_with_energy(self) -> float:
        w = C.c_double()
        if self._lib.oracle_step_with_energy(self._h, C.byref(w)) != 0:
            raise RuntimeError("oracle_step_with_energy failed")
        return w.value

    def field(self, field: int, axis: int) -> np.ndarray:
        out = np.empty(self.nodes, dtype=np.float32)
        if self._lib.oracle_download_field(self._h, field, axis, out.ctypes.data) != 0:
            raise RuntimeError("oracle_download_field failed")
        return out

    def set_field(self, field: int, axis: int, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float32)
        if self._lib.oracle_upload_field(self._h, field, axis, v.ctypes.data) != 0:
            raise RuntimeError("oracle_upload_field failed")

    def sample(self, sampler) -> np.ndarray:
        """The current state through an ``ems_b200.Sampler``: (points, 3) f64."""
        out = np.zeros((len(sampler), 3), dtype=np.float64)
        if self._lib.oracle_sample(self._h, sampler.table, out.ctypes.data) != 0:
            raise RuntimeError("oracle_sample failed")
        return out

    def samples(self, op: int, which: int = 0) -> np.ndarray:
        n = C.c_size_t()
        if self._lib.oracle_samples(self._h, op, which, None, 0, C.byref(n)) != 0:
            raise RuntimeError("oracle_samples failed")
        out = np.empty(n.value, dtype=np.float64)
        if n.value:
            self._lib.oracle_samples(self._h, op, which, out.ctypes.data, n.value, C.byref(n))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
