"""B200-native FDTD time stepping for ems, behind the reference engine's API.

The package mirrors the reference's engine-level interface
(src/engine/mod.rs ``EngineBuilder`` / ``Engine``, src/engine/boundary/cpml.rs
``CpmlBoundary``, src/engine/dispersive.rs ``Dispersive``, src/engine/port.rs
``LumpedPort``, src/engine/excite.rs ``EdgeSource``, src/engine/probe.rs
``Probe``, src/engine/run.rs ``run_until``): a :class:`Model` restates the
host-side set-up in C++ (``libems_host.so``) and hands the tables to the
CUDA engine (``libems_gpu.so``, :class:`Engine`). There is no CPU path: an
engine needs a CUDA device and raises if the CUDA library is missing.
"""
from __future__ import annotations

import ctypes as C
import cmath
import math
import os
from dataclasses import dataclass
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

# Face order x_min, x_max, y_min, y_max, z_min, z_max (src/fdtd.rs Face::ALL).
FACES = ("x_min", "x_max", "y_min", "y_max", "z_min", "z_max")
X, Y, Z = 0, 1, 2
SOFT_E, HARD_E, SOFT_H, HARD_H = 0, 1, 2, 3
VOLTAGE, CURRENT = 0, 1
PEC, PMC = 0, 1
LORENTZ, DRUDE, DEBYE, SHEET_BRANCH = 0, 1, 2, 3
# Pole schemes: trapezoidal, leapfrog, openEMS's f32 arithmetic (Lorentz and
# Drude poles take the material's own omega_p under it).
TRAPEZOIDAL, LEAPFROG, OPENEMS_POLES = 0, 1, 2
GAUSSIAN = 0

OP_CPML, OP_POLES, OP_LUMPED, OP_SOURCE, OP_PROBE, OP_MUR, OP_UPML, OP_SHEET = 1, 2, 3, 4, 5, 6, 7, 8
# Mur options (MurBoundary::openems_order / openems_corners / count_energy).
MUR_OPENEMS_ORDER, MUR_OPENEMS_CORNERS, MUR_COUNT_ENERGY = 1, 2, 4


# ems_status codes (include/ems_gpu.h).
ERR_INVALID, ERR_CUDA, ERR_DIVERGED, ERR_TIMEOUT, ERR_NOMEM = 1, 2, 3, 4, 5


class EngineError(RuntimeError):
    """An engine call failed; ``status`` is the ems_status code."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"ems status {status}: {msg}")
        self.status = status


# ----------------------------------------------------------------------------
# ctypes declarations of include/ems_gpu.h and include/ems_host.h


class FreqDumpSpec(C.Structure):
    """``ems_freq_dump`` (include/ems_gpu.h)."""

    _fields_ = [
        ("field", C.c_int32),
        ("lo", C.c_uint64 * 3),
        ("hi", C.c_uint64 * 3),
        ("stride", C.c_uint64 * 3),
        ("inv_len", C.c_void_p * 3),
        ("n_freqs", C.c_size_t),
        ("freqs", C.c_void_p),
        ("interval", C.c_uint64),
        ("sampler", C.c_void_p),
    ]


class TimeDumpSpec(C.Structure):
    """``ems_time_dump`` (include/ems_gpu.h)."""

    _fields_ = [("field", C.c_int32), ("lo", C.c_uint64 * 3), ("hi", C.c_uint64 * 3), ("stride", C.c_uint64 * 3),
                ("inv_len", C.c_void_p * 3), ("interval", C.c_uint64), ("sampler", C.c_void_p)]


class EngineDesc(C.Structure):
    _fields_ = [
        ("nodes", C.c_uint64 * 3),
        ("dt", C.c_double),
        ("coeff", C.c_void_p * 12),
        ("n_ops", C.c_size_t),
        ("ops", C.c_void_p),
    ]


class OpEntry(C.Structure):
    _fields_ = [("kind", C.c_int32), ("table", C.c_void_p)]


class CpmlSlab(C.Structure):
    _fields_ = [("e_side", C.c_int32), ("comp", C.c_int32), ("normal", C.c_int32), ("other", C.c_int32),
                ("sign", C.c_float), ("lo", C.c_uint64 * 3), ("hi", C.c_uint64 * 3),
                ("b", C.c_void_p), ("a", C.c_void_p), ("k", C.c_void_p)]


class CpmlTable(C.Structure):
    _fields_ = [("n_slabs", C.c_size_t), ("slabs", C.c_void_p)]


class PoleSide(C.Structure):
    _fields_ = [("n_edges", C.c_size_t), ("axis", C.c_void_p), ("node", C.c_void_p), ("sum_inv_z", C.c_void_p),
                ("pole_end", C.c_void_p), ("n_poles", C.c_size_t), ("kind", C.c_void_p), ("a", C.c_void_p),
                ("inv_c", C.c_void_p), ("inv_z", C.c_void_p), ("half_l", C.c_void_p)]


class PolesTable(C.Structure):
    _fields_ = [("electric", PoleSide), ("magnetic", PoleSide)]


class Stepper(C.Structure):
    _fields_ = [
        ("ctx", C.c_void_p),
        ("run", C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64)),
        ("step_with_energy", C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double))),
    ]


class BatchStepper(C.Structure):
    _fields_ = [
        ("ctx", C.c_void_p),
        ("n_models", C.c_size_t),
        ("run", C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64)),
        ("step_with_energy", C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double))),
        ("set_active", C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_size_t, C.c_int)),
    ]


class RunLimits(C.Structure):
    """``RunLimits`` (src/engine/run.rs:24-53) for :func:`run_until`."""

    _fields_ = [
        ("max_timesteps", C.c_uint64),
        ("has_end_criteria", C.c_int),
        ("energy_ratio", C.c_double),
        ("check_interval", C.c_uint64),
        ("has_excitation_end", C.c_int),
        ("excitation_end", C.c_double),
        ("dt", C.c_double),
    ]


class RunOutcome(C.Structure):
    """``RunOutcome`` (src/engine/run.rs:195-214); reason 0 energy decay,
    1 max timesteps, 2 diverged, 3 engine error."""

    _fields_ = [
        ("reason", C.c_int),
        ("steps", C.c_uint64),
        ("energy", C.c_double),
        ("max_energy", C.c_double),
        ("ratio_db", C.c_double),
        ("checks", C.c_uint64),
    ]


class UpmlTable(C.Structure):
    """``ems_upml`` (include/ems_gpu.h)."""

    _fields_ = [("n", C.c_size_t * 2), ("axis", C.c_void_p * 2), ("node", C.c_void_p * 2), ("co", C.c_void_p * 2)]


class MurTable(C.Structure):
    """``ems_mur`` (include/ems_gpu.h)."""

    _fields_ = [("n", C.c_size_t), ("n_edges", C.c_size_t), ("axis", C.c_void_p), ("node", C.c_void_p),
                ("inner", C.c_void_p), ("k", C.c_void_p), ("hold", C.c_void_p), ("cap", C.c_void_p),
                ("openems_order", C.c_int32), ("openems_corners", C.c_int32), ("count_energy", C.c_int32)]


_host = None
_gpu = None


def _u64(v: Sequence[int]):
    return (C.c_uint64 * len(v))(*[int(x) for x in v])


def _f64(v: Sequence[float]):
    return (C.c_double * len(v))(*[float(x) for x in v])


def host_lib() -> C.CDLL:
    """The host set-up library (built in-tree by ``ems_b200.build``)."""
    global _host
    if _host is None:
        path = os.path.join(HERE, "libems_host.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `python -m ems_b200.build`")
        L = C.CDLL(path)
        p, u, d, i, sz = C.c_void_p, C.c_uint64, C.c_double, C.c_int, C.c_size_t
        sig = {
            "ems_model_new": (p, [p, sz, p, sz, p, sz]),
            "ems_model_free": (None, [p]),
            "ems_model_error": (C.c_char_p, [p]),
            "ems_model_nodes": (None, [p, p]),
            "ems_model_material": (i, [p, p, p, p, p]),
            "ems_cellset_new": (p, [p]),
            "ems_cellset_free": (None, [p]),
            "ems_cellset_box": (i, [p, p, p]),
            "ems_cellset_sphere": (i, [p, p, d]),
            "ems_cellset_count": (u, [p]),
            "ems_model_fill": (i, [p, p, i]),
            "ems_model_pec_edges": (i, [p, i, p, p]),
            "ems_model_faces": (i, [p, p]),
            "ems_model_build": (i, [p, d, d]),
            "ems_model_build_bound": (i, [p, d, i]),
            "ems_model_openems_timestep": (d, [p, i]),
            "ems_model_zero_edges": (i, [p, i, i, p, p]),
            "ems_model_set_edge_circuit": (i, [p, i, p, d, d]),
            "ems_model_add_openems_pml": (i, [p, p]),
            "ems_model_set_edge_materials": (i, [p, i, i, p, p]),
            "ems_model_set_mur_media": (i, [p, i, i, p]),
            "ems_model_dt": (d, [p]),
            "ems_model_courant_limit": (d, [p]),
            "ems_model_coeff": (p, [p, i]),
            "ems_model_add_cpml": (i, [p, p, d, d, d, d, i]),
            "ems_model_cpml_index": (d, [p, i]),
            "ems_dispersive_new": (p, []),
            "ems_dispersive_free": (None, [p]),
            "ems_dispersive_fill": (i, [p, p, p, i, sz, p, p, p, p]),
            "ems_model_add_dispersive": (i, [p, p, i]),
            "ems_dispersive_add_edge": (i, [p, i, i, p, i, d, d, d]),
            "ems_model_edge_material": (i, [p, i, i, p, p]),
            "ems_waveform_value": (d, [i, d, d, d, d]),
            "ems_waveform_duration": (d, [i, d, d]),
            "ems_model_add_lumped_port": (i, [p, i, p, p, d, i, d, d, d, u]),
            "ems_model_add_lumped": (i, [p, i, p, p, d, d, d, i, i, i, p, u]),
            "ems_model_add_lumped_openems": (i, [p, i, p, p, d, d, d, i, d, i, p, p, u]),
            "ems_model_add_absorbing_sheet": (i, [p, i, u, i, p, p, d, i]),
            "ems_model_add_source": (i, [p, i, sz, p, p, p, i, d, d, u]),
            "ems_model_add_source_table": (i, [p, i, sz, p, p, p, p, u]),
            "ems_model_add_probe": (i, [p, i, sz, p, p, p, u]),
            "ems_model_add_mur": (i, [p, p, p, p, i]),
            "ems_model_add_sheet": (i, [p, sz, p, p, p, p, p, p, p, d, p, p]),
            "ems_sheet_layer_profile": (sz, [d, d, d, p, sz]),
            "ems_sampler_new": (p, [p, i, i, p, p, p]),
            "ems_sampler_new_indices": (p, [p, i, i, p, p]),
            "ems_sampler_table": (p, [p]),
            "ems_sampler_coords": (p, [p, i, p]),
            "ems_sampler_free": (None, [p]),
            "ems_model_probe_f32": (i, [p, i, i]),
            "ems_model_desc": (p, [p]),
            "ems_dft": (None, [d, d, p, sz, p, sz, p, p]),
            "ems_drive": (i, [p, p, p]),
            "ems_batch_drive": (i, [p, p, p]),
            "ems_const_eps0": (d, []),
            "ems_const_mu0": (d, []),
            "ems_const_c0": (d, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _host = L
    return _host


GPU_SYMBOLS = {
    "ems_gpu_create": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "ems_gpu_destroy": (C.c_int, [C.c_void_p]),
    "ems_gpu_run": (C.c_int, [C.c_void_p, C.c_uint64]),
    "ems_gpu_step_with_energy": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ems_gpu_timestep": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ems_gpu_download_field": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "ems_gpu_upload_field": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "ems_gpu_samples": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]),
    "ems_gpu_last_error": (C.c_char_p, [C.c_void_p]),
    "ems_gpu_launch_count": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ems_gpu_set_schedule": (C.c_int, [C.c_void_p, C.c_int]),
    "ems_gpu_set_curl_order": (C.c_int, [C.c_void_p, C.c_int]),
    "ems_gpu_time_dump_add": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "ems_gpu_upml_state": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_void_p, C.c_void_p, C.c_size_t]),
    "ems_gpu_time_dump_count": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p]),
    "ems_gpu_time_dump_read": (C.c_int, [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p]),
    "ems_gpu_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ems_gpu_schedule": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ems_gpu_interior_box": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ems_gpu_row_cpml": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ems_gpu_set_row_cpml": (C.c_int, [C.c_void_p, C.c_int]),
    "ems_energy_noalloc": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]),
    "ems_gpu_last_sample": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_void_p]),
    "ems_gpu_source_amplitude": (C.c_int, [C.c_void_p, C.c_size_t, C.c_uint64, C.c_void_p, C.c_size_t]),
    "ems_gpu_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "ems_gpu_profile_read": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "ems_gpu_autotune": (C.c_int, [C.c_void_p, C.c_char_p]),
    "ems_gpu_freq_dump_add": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "ems_gpu_set_sweep_planes": (C.c_int, [C.c_void_p, C.c_uint32]),
    "ems_gpu_set_interior_planes": (C.c_int, [C.c_void_p, C.c_uint32]),
    "ems_gpu_set_march": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32]),
    "ems_gpu_check": (C.c_int, [C.c_void_p]),
    "ems_gpu_test_wait_timeout": (C.c_int, [C.c_void_p, C.c_uint64]),
    "ems_gpu_freq_dump_read": (C.c_int, [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_size_t]),
    "ems_batch_autotune": (C.c_int, [C.c_void_p, C.c_char_p]),
    "ems_batch_create": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_uint64, C.c_void_p]),
    "ems_batch_destroy": (C.c_int, [C.c_void_p]),
    "ems_batch_run": (C.c_int, [C.c_void_p, C.c_uint64]),
    "ems_batch_step_with_energy": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ems_batch_set_active": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int]),
    "ems_batch_timestep": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p]),
    "ems_batch_samples": (C.c_int, [C.c_void_p, C.c_size_t, C.c_size_t, C.c_int, C.c_void_p, C.c_size_t,
                                    C.c_void_p]),
    "ems_batch_download_field": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_void_p]),
    "ems_batch_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ems_batch_last_error": (C.c_char_p, [C.c_void_p]),
}


def gpu_lib() -> C.CDLL:
    """The CUDA engine library. Raises if it is missing: there is no CPU path."""
    global _gpu
    if _gpu is None:
        path = os.path.join(HERE, "libems_gpu.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: the CUDA engine is not built (python -m ems_b200.build)")
        L = C.CDLL(path)
        for name, (res, args) in GPU_SYMBOLS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _gpu = L
    return _gpu


def eps0() -> float:
    return host_lib().ems_const_eps0()


def mu0() -> float:
    return host_lib().ems_const_mu0()


def c0() -> float:
    return host_lib().ems_const_c0()


def waveform_value(f0: float, fc: float, t: float, dt: float = 0.0) -> float:
    """``Waveform::Gaussian{f0, fc}.value(t, dt)`` (src/waveform.rs:455-463)."""
    return host_lib().ems_waveform_value(GAUSSIAN, f0, fc, t, dt)


def waveform_duration(f0: float, fc: float) -> float:
    """``Waveform::duration``: 2T of the Gaussian (src/waveform.rs:485-492)."""
    return host_lib().ems_waveform_duration(GAUSSIAN, f0, fc)


# ----------------------------------------------------------------------------
# host-side model (the reference's EngineBuilder + operator set-up)


class CellSet:
    """A set of cells (boxes, spheres) for materials and dispersive media."""

    def __init__(self, model: "Model"):
        self._lib = host_lib()
        self._p = self._lib.ems_cellset_new(model._p)

    def box(self, lo: Sequence[int], hi: Sequence[int]) -> "CellSet":
        if self._lib.ems_cellset_box(self._p, _u64(lo), _u64(hi)) != 0:
            raise ValueError(f"cell box {lo}..{hi} outside the grid")
        return self

    def sphere(self, centre: Sequence[float], radius: float) -> "CellSet":
        self._lib.ems_cellset_sphere(self._p, _f64(centre), float(radius))
        return self

    def count(self) -> int:
        return int(self._lib.ems_cellset_count(self._p))

    def __del__(self):
        if getattr(self, "_p", None):
            self._lib.ems_cellset_free(self._p)
            self._p = None


@dataclass
class Pole:
    """``Pole`` (src/engine/dispersive.rs:211-244), frequencies in rad/s."""

    kind: int
    p1: float
    p2: float = 0.0
    p3: float = 0.0

    @staticmethod
    def lorentz(omega_p: float, omega_0: float, gamma: float) -> "Pole":
        return Pole(LORENTZ, omega_p, omega_0, gamma)

    @staticmethod
    def drude(omega_p: float, gamma: float) -> "Pole":
        return Pole(DRUDE, omega_p, gamma)

    @staticmethod
    def debye(delta_eps: float, tau: float) -> "Pole":
        return Pole(DEBYE, delta_eps, tau)

    @staticmethod
    def sheet_branch(inductance: float, resistance: float) -> "Pole":
        """A series R-L branch of openEMS's conducting-sheet model on one E
        edge (src/engine/openems_sheet.rs), for ``Dispersive.add_edge``
        with the openEMS pole scheme."""
        return Pole(SHEET_BRANCH, inductance, resistance)


class Dispersive:
    """``Dispersive`` (src/engine/dispersive.rs:1800-1985): collect poles
    with :meth:`fill_cells`, install with :meth:`Model.add_dispersive`."""

    def __init__(self):
        self._lib = host_lib()
        self._p = self._lib.ems_dispersive_new()

    def fill_cells(self, model: "Model", cells: CellSet, poles: Sequence[Pole], field: int = 0) -> "Dispersive":
        n = len(poles)
        kinds = (C.c_int * n)(*[p.kind for p in poles])
        r = self._lib.ems_dispersive_fill(self._p, model._p, cells._p, field, n, kinds,
                                          _f64([p.p1 for p in poles]), _f64([p.p2 for p in poles]),
                                          _f64([p.p3 for p in poles]))
        if r != 0:
            raise ValueError("invalid dispersive pole")
        return self

    def add_edge(self, field: int, axis: int, node: Sequence[int], pole: "Pole") -> "Dispersive":
        """One full (unscaled) pole on the E edge (field 0) or H dual edge
        (field 1) along ``axis`` at ``node``."""
        r = self._lib.ems_dispersive_add_edge(self._p, field, axis, _u64(node), pole.kind, pole.p1, pole.p2, pole.p3)
        if r != 0:
            raise ValueError("invalid dispersive pole")
        return self

    def __del__(self):
        if getattr(self, "_p", None):
            self._lib.ems_dispersive_free(self._p)
            self._p = None


class Model:
    """A compiled model: grid, materials, coefficients and operator tables.

    Restates ``Engine::builder(grid).materials(m).faces(f).timestep(t).build()``
    and the operators' set-up (src/engine/mod.rs:325-381) on the host.
    """

    def __init__(self, x: Sequence[float], y: Sequence[float], z: Sequence[float]):
        self._lib = host_lib()
        self._keep = [np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z)]
        a = self._keep
        self._p = self._lib.ems_model_new(a[0].ctypes.data, len(a[0]), a[1].ctypes.data, len(a[1]),
                                          a[2].ctypes.data, len(a[2]))
        if not self._p:
            raise ValueError("invalid grid lines (need >= 2 strictly increasing finite lines per axis)")
        self.ops: list[tuple[int, str]] = []

    @staticmethod
    def uniform(cells: Sequence[int], size: Sequence[float]) -> "Model":
        """``Grid::uniform`` (src/engine/grid.rs:514-519)."""
        return Model(*[np.arange(cells[a] + 1, dtype=np.float64) * size[a] for a in range(3)])

    def _check(self, r: int, what: str) -> int:
        if r < 0 or (what.endswith("!") and r != 0):
            raise ValueError(f"{what.rstrip('!')}: {self._lib.ems_model_error(self._p).decode()}")
        return r

    @property
    def nodes(self) -> tuple[int, int, int]:
        n = (C.c_uint64 * 3)()
        self._lib.ems_model_nodes(self._p, n)
        return (int(n[0]), int(n[1]), int(n[2]))

    def material(self, eps_r=1.0, mu_r=1.0, kappa=0.0, sigma_m=0.0) -> int:
        """``Material`` (src/engine/material.rs): scalars or per-axis triples."""
        v = lambda x: _f64(list(x) if hasattr(x, "__len__") else [x] * 3)  # noqa: E731
        return self._check(self._lib.ems_model_material(self._p, v(eps_r), v(mu_r), v(kappa), v(sigma_m)), "material")

    def cells(self) -> CellSet:
        return CellSet(self)

    def inv_edge_lengths(self, axis: int, dual: bool = False) -> np.ndarray:
        """1/length of the edges along `axis` per node index: primary edges
        (``Grid::delta``; 0 at the last node, which starts no edge) or dual
        edges (``Grid::dual_delta``: half a cell on the outer nodes)."""
        x = self._keep[axis]
        d = np.diff(x)
        n = len(x)
        if dual:
            dd = np.empty(n)
            dd[0], dd[-1] = 0.5 * d[0], 0.5 * d[-1]
            dd[1:-1] = 0.5 * (d[:-1] + d[1:])
            return 1.0 / dd
        out = np.zeros(n)
        out[:-1] = 1.0 / d
        return out

    def fill(self, cells: CellSet, mat: int) -> "Model":
        self._check(self._lib.ems_model_fill(self._p, cells._p, mat), "fill!")
        return self

    def pec_edges(self, axis: int, lo: Sequence[int], hi: Sequence[int]) -> "Model":
        self._check(self._lib.ems_model_pec_edges(self._p, axis, _u64(lo), _u64(hi)), "pec_edges!")
        return self

    def fill_pec_box(self, lo: Sequence[int], hi: Sequence[int]) -> "Model":
        """``CellMaterials::fill_pec_box`` over the node ranges lo..hi (half-open):
        every edge of every axis with both ends in the box."""
        for a in range(3):
            top = [h - 1 for h in hi]
            top[a] = hi[a] - 2
            if top[a] >= lo[a] and all(top[t] >= lo[t] for t in range(3)):
                self.pec_edges(a, lo, top)
        return self

    def faces(self, faces: Sequence[int]) -> "Model":
        self._check(self._lib.ems_model_faces(self._p, (C.c_int * 6)(*faces)), "faces!")
        return self

    def build(self, courant: float = 0.99, dt: float | None = None) -> "Model":
        self._check(self._lib.ems_model_build(self._p, courant, 0.0 if dt is None else dt), "build!")
        return self

    def set_edge_materials(self, field: int, axis: int, v0: np.ndarray, v1: np.ndarray) -> "Model":
        """Per-edge (eps_r, kappa) of the E edges (field 0) or (mu_r,
        sigma_m) of the H dual edges (field 1) along ``axis``, node arrays,
        in place of the cell averages (before build)."""
        a0 = np.ascontiguousarray(v0, dtype=np.float64).ravel()
        a1 = np.ascontiguousarray(v1, dtype=np.float64).ravel()
        self._check(self._lib.ems_model_set_edge_materials(self._p, field, axis, a0.ctypes.data, a1.ctypes.data),
                    "set_edge_materials!")
        return self

    def set_mur_media(self, face: int, axis: int, v: np.ndarray) -> "Model":
        """Phase velocities of the edges along ``axis`` on Mur ``face`` (0
        x_min … 5 z_max), a (n_u, n_w) array over the face plane (u < w the
        other axes; 0 keeps the local medium); before ``add_mur``."""
        a = np.ascontiguousarray(v, dtype=np.float64).ravel()
        self._check(self._lib.ems_model_set_mur_media(self._p, face, axis, a.ctypes.data), "set_mur_media!")
        return self

    def build_bound(self, dt: float, openems_rounding: bool = False, openems_sigma_m: bool = False) -> "Model":
        """Builds with ``dt`` as given (``TimeStep::Bound``), the exact or
        openEMS coefficient rounding (``CoeffRounding``) and csx's or
        openEMS's average of the magnetic conductivity."""
        flags = (1 if openems_rounding else 0) | (2 if openems_sigma_m else 0)
        self._check(self._lib.ems_model_build_bound(self._p, dt, flags), "build_bound!")
        return self

    def openems_timestep(self, method: int = 3) -> float:
        """openEMS's time step (``TimeStepMethod`` 3 Rennings, 1 CFL) of
        the grid and materials (src/engine/timestep.rs)."""
        dt = self._lib.ems_model_openems_timestep(self._p, method)
        if not dt > 0.0:
            raise ValueError(f"unknown time-step method {method}")
        return dt

    def set_edge_circuit(self, axis: int, node: Sequence[int], cap: float = -1.0, cond: float = -1.0) -> "Model":
        """Replaces an E edge's capacitance and/or conductance (negative:
        the medium's) after build."""
        self._check(self._lib.ems_model_set_edge_circuit(self._p, axis, _u64(node), cap, cond), "set_edge_circuit!")
        return self

    def zero_edges(self, field: int, axis: int, lo: Sequence[int], hi: Sequence[int]) -> "Model":
        """Zeroes the coefficients of the E (field 0) or H (1) edges along
        ``axis`` at the nodes of the inclusive box lo..hi (after build)."""
        self._check(self._lib.ems_model_zero_edges(self._p, field, axis, _u64(lo), _u64(hi)), "zero_edges!")
        return self

    @property
    def dt(self) -> float:
        return self._lib.ems_model_dt(self._p)

    @property
    def courant_limit(self) -> float:
        return self._lib.ems_model_courant_limit(self._p)

    def coeff(self, lane: int) -> np.ndarray:
        """Coefficient lane (ca 0-2, cb 3-5, da 6-8, db 9-11), reference layout (a copy)."""
        n = int(np.prod(self.nodes))
        p = self._lib.ems_model_coeff(self._p, lane)
        return np.ctypeslib.as_array((C.c_float * n).from_address(p)).copy().reshape(self.nodes)

    def add_cpml(self, cells: Sequence[int], grading: float = 3.0, sigma_factor: float = 1.0,
                 kappa_max: float = 1.0, alpha_max: float = 0.0, linear: bool = True) -> int:
        """``CpmlBoundary::new(engine, faces)`` (src/engine/boundary/cpml.rs:941-951)."""
        r = self._check(self._lib.ems_model_add_cpml(self._p, _u64(cells), grading, sigma_factor, kappa_max,
                                                     alpha_max, 1 if linear else 0), "add_cpml")
        self.ops.append((OP_CPML, "cpml"))
        return r

    def cpml_index(self, face: int) -> float:
        return self._lib.ems_model_cpml_index(self._p, face)

    def add_dispersive(self, d: Dispersive, scheme: int = TRAPEZOIDAL) -> int:
        r = self._check(self._lib.ems_model_add_dispersive(self._p, d._p, scheme), "add_dispersive")
        self.ops.append((OP_POLES, "poles"))
        return r

    def add_lumped_port(self, axis: int, lo: Sequence[int], hi: Sequence[int], r: float, f0: float, fc: float,
                        amplitude: float, n_steps: int) -> int:
        """``LumpedPort::new(LumpedBox(axis, lo, hi), r).excite_waveform(Gaussian{f0, fc}, amplitude)``."""
        k = self._check(self._lib.ems_model_add_lumped_port(self._p, axis, _u64(lo), _u64(hi), r, GAUSSIAN, f0, fc,
                                                            amplitude, n_steps), "add_lumped_port")
        self.ops.append((OP_LUMPED, "port"))
        return k

    def add_lumped_port_table(self, axis: int, lo: Sequence[int], hi: Sequence[int], r: float,
                              amp: np.ndarray | None) -> int:
        """``LumpedPort::new(LumpedBox(axis, lo, hi), r).excite(v)`` with ``amp[n]`` = v((n + ½)·dt)
        (src/engine/port.rs:102-155); ``amp`` None: a passive port."""
        return self.add_lumped(axis, lo, hi, r=r, amp=amp, port=True)

    def add_lumped(self, axis: int, lo: Sequence[int], hi: Sequence[int], r: float = 0.0, l: float = 0.0,
                   c: float = 0.0, series: bool = False, record: bool = False, port: bool = False,
                   amp: np.ndarray | None = None) -> int:
        """``LumpedElement::new(LumpedBox(axis, lo, hi)).r(r).l(l).c(c)`` (0: absent) with the
        parallel or series topology, optionally ``record_current()`` and a Thevenin source
        sampled at (n + ½)·dt (src/engine/lumped.rs:380-1013)."""
        a = None if amp is None else np.ascontiguousarray(amp, dtype=np.float64)
        k = self._check(self._lib.ems_model_add_lumped(self._p, axis, _u64(lo), _u64(hi), r, l, c, int(series),
                                                       int(record), int(port),
                                                       None if a is None else a.ctypes.data,
                                                       0 if a is None else len(a)), "add_lumped")
        self.ops.append((OP_LUMPED, "port" if port else "lumped"))
        return k

    def add_lumped_openems(self, axis: int, lo: Sequence[int], hi: Sequence[int], r: float = 0.0, l: float = 0.0,
                           c: float = 0.0, series: bool = False, omega: float = 0.0, explicit: bool = True,
                           src_w: np.ndarray | None = None, amp: np.ndarray | None = None) -> int:
        """A lumped element with an inductor or in series as an openEMS file has it
        (``ems_model_add_lumped_openems``; src/sim/map.rs:820-1000, 1525-1632): the
        element replaces the medium of its edges, the edge capacitance is limited at
        ``omega``, openEMS's order and (parallel inductor, ``explicit``) its explicit
        f32 update; ``src_w`` (per edge) and ``amp`` (at (n + ½)·dt) its Thevenin
        source (a parallel element with a resistor)."""
        w = None if src_w is None else np.ascontiguousarray(src_w, dtype=np.float64)
        a = None if amp is None else np.ascontiguousarray(amp, dtype=np.float64)
        k = self._check(self._lib.ems_model_add_lumped_openems(
            self._p, axis, _u64(lo), _u64(hi), r, l, c, int(series), omega, int(explicit),
            None if w is None else w.ctypes.data, None if a is None else a.ctypes.data,
            0 if a is None else len(a)), "add_lumped_openems")
        self.ops.append((OP_LUMPED, "lumped"))
        return k

    def add_absorbing_sheet(self, normal: int, plane: int, positive: bool, start: Sequence[int],
                            stop: Sequence[int], velocity: float = 0.0, openems_order: bool = False) -> int:
        """``AbsorbingSheet::new(engine, AbcSheet{..}, velocity)`` (src/engine/boundary/abc.rs):
        first-order Mur on the tangential E edges of the rectangle start..stop on mesh
        plane ``plane`` normal to ``normal``, absorbing waves along +normal (``positive``)
        or -normal; ``velocity`` <= 0: the local medium velocity per edge."""
        k = self._check(self._lib.ems_model_add_absorbing_sheet(self._p, normal, plane, int(positive), _u64(start),
                                                                _u64(stop), velocity, int(openems_order)),
                        "add_absorbing_sheet")
        self.ops.append((OP_MUR, "abc"))
        return k

    def add_sheet(self, edges: Sequence[tuple], f_max: float | None = None) -> int:
        """``ConductingSheet::new(f_max)``, ``push(SheetEdge{..})`` per edge, ``add_to``
        (src/engine/sheet.rs:529-935): each edge is ``(axis, node, normal, sigma, thickness)``
        or with ``upper_share=(c, g)`` appended. ``f_max`` None: 1/(10·dt). Sets
        ``sheet_edges`` / ``sheet_skipped`` (PEC edges and duplicates) of the returned op."""
        n = len(edges)
        axis = (C.c_int * max(n, 1))(*[e[0] for e in edges])
        nodes = _u64([c for e in edges for c in e[1]] or [0])
        normal = (C.c_int * max(n, 1))(*[e[2] for e in edges])
        sig = _f64([e[3] for e in edges] or [0.0])
        th = _f64([e[4] for e in edges] or [0.0])
        sc = _f64([(e[5][0] if len(e) > 5 and e[5] is not None else -1.0) for e in edges] or [0.0])
        sg = _f64([(e[5][1] if len(e) > 5 and e[5] is not None else -1.0) for e in edges] or [0.0])
        inst, skip = C.c_uint64(0), C.c_uint64(0)
        k = self._check(self._lib.ems_model_add_sheet(self._p, n, axis, nodes, normal, sig, th, sc, sg,
                                                      0.0 if f_max is None else float(f_max),
                                                      C.byref(inst), C.byref(skip)), "add_sheet")
        self.ops.append((OP_SHEET, "sheet"))
        self.sheet_edges = getattr(self, "sheet_edges", {})
        self.sheet_edges[k] = (int(inst.value), int(skip.value))
        return k

    def add_sheet_rect(self, normal: int, plane: int, start: Sequence[int], stop: Sequence[int], sigma: float,
                       t: float, f_max: float | None = None) -> int:
        """``ConductingSheet::add_rect`` (src/engine/sheet.rs:573-603) then ``add_to``: every
        tangential edge of the node rectangle start..=stop on node plane ``plane``."""
        return self.add_sheet(sheet_rect_edges(normal, plane, start, stop, sigma, t), f_max)

    def add_source(self, kind: int, edges: Sequence[tuple[int, Sequence[int], float]], f0: float, fc: float,
                   n_steps: int) -> int:
        """``EdgeSource::new(|t| Gaussian{f0, fc}.value(t)).kind(kind).edge(axis, node, w)...``"""
        n = len(edges)
        axis = (C.c_int * n)(*[e[0] for e in edges])
        nodes = _u64([c for e in edges for c in e[1]])
        w = _f64([e[2] for e in edges])
        k = self._check(self._lib.ems_model_add_source(self._p, kind, n, axis, nodes, w, GAUSSIAN, f0, fc, n_steps),
                        "add_source")
        self.ops.append((OP_SOURCE, "source"))
        return k

    def add_source_table(self, kind: int, edges: Sequence[tuple[int, Sequence[int], float]],
                         amplitude: np.ndarray) -> int:
        """``EdgeSource::new(f)`` with f sampled by the caller: ``amplitude[n]``
        is f at the kind's sample time of step n ((n+½)dt for soft E)."""
        n = len(edges)
        axis = (C.c_int * n)(*[e[0] for e in edges])
        nodes = _u64([c for e in edges for c in e[1]])
        w = _f64([e[2] for e in edges])
        amp = np.ascontiguousarray(amplitude, dtype=np.float64)
        k = self._check(self._lib.ems_model_add_source_table(self._p, kind, n, axis, nodes, w, amp.ctypes.data,
                                                             len(amp)), "add_source_table")
        self.ops.append((OP_SOURCE, "source"))
        return k

    def add_source_arrays(self, kind: int, axis: np.ndarray, nodes: np.ndarray, weight: np.ndarray, f0: float,
                          fc: float, n_steps: int) -> int:
        """:meth:`add_source` from arrays (n axes, n×3 nodes, n weights)."""
        axis = np.ascontiguousarray(axis, dtype=np.int32)
        nodes = np.ascontiguousarray(nodes, dtype=np.uint64)
        weight = np.ascontiguousarray(weight, dtype=np.float64)
        k = self._check(self._lib.ems_model_add_source(self._p, kind, len(axis), axis.ctypes.data, nodes.ctypes.data,
                                                       weight.ctypes.data, GAUSSIAN, f0, fc, n_steps), "add_source")
        self.ops.append((OP_SOURCE, "source"))
        return k

    def add_mur(self, faces, hold: dict | None = None, flags: int = 0) -> int:
        """``MurBoundary::with_faces_in(engine, faces, materials)``
        (src/engine/boundary/mur.rs:355-401): ``faces`` maps a face (index or
        name) to its phase velocity in m/s, or to None for each edge's local
        medium speed; ``hold`` maps faces to the step before which their
        edges are not updated (``hold_faces``); flags: MUR_* bits."""
        mode = (C.c_int * 6)()
        vel = (C.c_double * 6)()
        for f, v in dict(faces).items():
            f = FACES.index(f) if isinstance(f, str) else int(f)
            mode[f] = 2 if v is None else 1
            vel[f] = 0.0 if v is None else float(v)
        held = None
        if hold:
            h = [0] * 6
            for f, until in hold.items():
                h[FACES.index(f) if isinstance(f, str) else int(f)] = int(until)
            held = _u64(h)
        k = self._check(self._lib.ems_model_add_mur(self._p, mode, vel, held, int(flags)), "add_mur")
        self.ops.append((OP_MUR, "mur"))
        return k

    def add_probe(self, quantity: int, entries: Sequence[tuple[int, Sequence[int], float]], interval: int = 1,
                  f32_sum: bool = False) -> int:
        """``Probe::new(quantity).entry(axis, node, w)...interval(n)`` (src/engine/probe.rs);
        ``f32_sum``: entries summed in f32, as openEMS's current probes."""
        n = len(entries)
        axis = (C.c_int * n)(*[e[0] for e in entries])
        nodes = _u64([c for e in entries for c in e[1]])
        w = _f64([e[2] for e in entries])
        k = self._check(self._lib.ems_model_add_probe(self._p, quantity, n, axis, nodes, w, interval), "add_probe")
        self.ops.append((OP_PROBE, "probe"))
        if f32_sum:
            self._check(self._lib.ems_model_probe_f32(self._p, k, 1), "probe_f32!")
        return k

    @property
    def desc(self) -> int:
        """Address of the ems_engine_desc (valid while the model is alive and unchanged)."""
        p = self._lib.ems_model_desc(self._p)
        if not p:
            raise ValueError("model not built")
        return p

    def edge_material(self, field: int, axis: int, node: Sequence[int]) -> tuple[float, float]:
        """(eps_r, kappa) of an E edge (field 0) or (mu_r, sigma_m) of an H
        dual edge (field 1), averaged over its cells (EdgeMaterials)."""
        out = (C.c_double * 2)()
        if self._lib.ems_model_edge_material(self._p, field, axis, _u64(node), out) != 0:
            raise ValueError("edge outside the grid")
        return out[0], out[1]

    def add_openems_pml(self, cells: Sequence[int]) -> int:
        """openEMS's ``PML_n`` layers of ``cells[f]`` cells on face f
        (``OpenEmsPml``, src/engine/boundary/upml.rs): rewrites the layer
        edges' coefficients and adds the layer operator."""
        k = self._check(self._lib.ems_model_add_openems_pml(self._p, _u64(cells)), "add_openems_pml")
        self.ops.append((OP_UPML, "upml"))
        return k

    def upml_table(self, op: int) -> list:
        """Per side (0 E, 1 H): (axis, node as (i, j, k), co (n, 4)) of the
        openEMS PML operator ``op`` (copies)."""
        d = EngineDesc.from_address(self.desc)
        ops = (OpEntry * d.n_ops).from_address(d.ops) if d.n_ops else []
        if not 0 <= op < d.n_ops or ops[op].kind != OP_UPML:
            raise ValueError("not an openEMS PML operator")
        t = UpmlTable.from_address(ops[op].table)
        ny, nz = self.nodes[1], self.nodes[2]
        out = []
        for sd in range(2):
            n = int(t.n[sd])
            if not n:
                out.append((np.zeros(0, np.int64), np.zeros((0, 3), np.int64), np.zeros((0, 4), np.float32)))
                continue
            ax = np.ctypeslib.as_array((C.c_uint8 * n).from_address(t.axis[sd])).astype(np.int64)
            flat = np.ctypeslib.as_array((C.c_uint64 * n).from_address(t.node[sd])).astype(np.int64)
            co = np.ctypeslib.as_array((C.c_float * (4 * n)).from_address(t.co[sd])).reshape(n, 4).copy()
            out.append((ax, np.stack([flat // (ny * nz), (flat // nz) % ny, flat % nz], axis=-1), co))
        return out

    def mur_table(self, op: int) -> dict:
        """The Mur operator ``op``'s entries as handed to the engine (copies):
        axis, node/inner as (i, j, k), k (2 per entry), hold, cap, and the
        number of face edges (the rest are edges shared by two faces)."""
        d = EngineDesc.from_address(self.desc)
        ops = (OpEntry * d.n_ops).from_address(d.ops) if d.n_ops else []
        if not 0 <= op < d.n_ops or ops[op].kind != OP_MUR:
            raise ValueError("not a Mur operator")
        t = MurTable.from_address(ops[op].table)
        n = int(t.n)
        ny, nz = self.nodes[1], self.nodes[2]

        def arr(ptr, ctype, count, dtype):
            if not ptr or not count:
                return np.zeros(count, dtype=dtype)
            return np.ctypeslib.as_array((ctype * count).from_address(ptr)).astype(dtype)

        def ijk(flat):
            return np.stack([flat // (ny * nz), (flat // nz) % ny, flat % nz], axis=-1)

        return {
            "n_edges": int(t.n_edges),
            "axis": arr(t.axis, C.c_uint8, n, np.int64),
            "node": ijk(arr(t.node, C.c_uint64, n, np.int64)),
            "inner": ijk(arr(t.inner, C.c_uint64, 2 * n, np.int64)).reshape(n, 2, 3),
            "k": arr(t.k, C.c_float, 2 * n, np.float32).reshape(n, 2),
            "hold": arr(t.hold, C.c_uint64, n, np.int64),
            "cap": arr(t.cap, C.c_double, n, np.float64),
        }

    def __del__(self):
        if getattr(self, "_p", None):
            self._lib.ems_model_free(self._p)
            self._p = None


# ----------------------------------------------------------------------------
# the CUDA engine


class Engine:
    """The CUDA engine for a built :class:`Model` (``Engine``, src/engine/mod.rs)."""

    def __init__(self, model: Model, device: int = 0):
        self._lib = gpu_lib()
        self._model = model
        h = C.c_void_p()
        st = self._lib.ems_gpu_create(model.desc, device, C.byref(h))
        if st != 0:
            raise EngineError(st, "ems_gpu_create failed")
        self._h = h
        self.nodes = model.nodes
        self.dt = model.dt

    def _ck(self, st: int) -> None:
        if st != 0:
            raise EngineError(st, self._lib.ems_gpu_last_error(self._h).decode())

    def run(self, n: int) -> None:
        self._ck(self._lib.ems_gpu_run(self._h, n))

    def step_with_energy(self) -> float:
        w = C.c_double()
        self._ck(self._lib.ems_gpu_step_with_energy(self._h, C.byref(w)))
        return w.value

    @property
    def timestep(self) -> int:
        n = C.c_uint64()
        self._ck(self._lib.ems_gpu_timestep(self._h, C.byref(n)))
        return n.value

    @property
    def launches(self) -> int:
        n = C.c_uint64()
        self._ck(self._lib.ems_gpu_launch_count(self._h, C.byref(n)))
        return n.value

    def set_curl_order(self, order: int) -> None:
        """0 the reference's default summation order of the curl, 1
        openEMS's (``CurlOrder``; per-operator, split and sweep schedules)."""
        self._ck(self._lib.ems_gpu_set_curl_order(self._h, order))

    def set_schedule(self, s: int) -> None:
        """0 automatic, 1 per-operator kernels, 2 fused single pass, 3 two
        kernels, 4 split, 5 sweep, 6 interior (one pass inside the CPML)."""
        self._ck(self._lib.ems_gpu_set_schedule(self._h, s))

    @property
    def schedule(self) -> int:
        """The schedule steps run with: 1 per-operator kernels, 2 fused, 3 two kernels, 4 split, 5 sweep,
        6 interior."""
        v = C.c_int()
        self._ck(self._lib.ems_gpu_schedule(self._h, C.byref(v)))
        return v.value

    def set_row_cpml(self, on: bool) -> None:
        """The split schedule's row CPML on or off (``ems_gpu_set_row_cpml``)."""
        self._ck(self._lib.ems_gpu_set_row_cpml(self._h, int(on)))

    @property
    def row_cpml(self) -> bool:
        """Whether split steps apply the CPML inside the update kernels (no shell kernel)."""
        v = C.c_int()
        self._ck(self._lib.ems_gpu_row_cpml(self._h, C.byref(v)))
        return bool(v.value)

    @property
    def interior_box(self) -> tuple:
        """The interior schedule's box: nodes (lo, hi) per axis."""
        b = (C.c_uint32 * 6)()
        self._ck(self._lib.ems_gpu_interior_box(self._h, b))
        return tuple(b[:3]), tuple(b[3:])

    def set_interior_planes(self, planes: int) -> None:
        """Planes a block of the interior schedule's one-pass kernel marches through."""
        self._ck(self._lib.ems_gpu_set_interior_planes(self._h, planes))

    def check(self) -> None:
        """Raises EngineError with EMS_ERR_TIMEOUT or EMS_ERR_DIVERGED if the
        device flags were set since the last check (``ems_gpu_check``)."""
        self._ck(self._lib.ems_gpu_check(self._h))

    def test_wait_timeout(self, limit_ns: int) -> None:
        """Arms the bounded-wait test hook for the next marching step."""
        self._ck(self._lib.ems_gpu_test_wait_timeout(self._h, limit_ns))

    def set_march(self, shape: int = 0, planes: int = 32) -> None:
        """The marching schedule's tile shape (0..3) and planes per block."""
        self._ck(self._lib.ems_gpu_set_march(self._h, shape, planes))

    def set_sweep_planes(self, planes: int) -> None:
        """Chunk size of the sweep schedule (5), in x-planes."""
        self._ck(self._lib.ems_gpu_set_sweep_planes(self._h, planes))

    def add_freq_dump(self, field: int, lo, hi, freqs, stride=(1, 1, 1), interval: int = 1) -> int:
        """A running DFT of E (field 0) or H (field 1) over the node box
        lo..hi (inclusive) on the device (``ems_gpu_freq_dump_add``); the
        edge lengths come from the model's lines. Returns the dump id."""
        m = self._model
        inv = [m.inv_edge_lengths(a, dual=field == 1) for a in range(3)]
        fr = np.ascontiguousarray(freqs, dtype=np.float64)
        spec = FreqDumpSpec(field, (C.c_uint64 * 3)(*lo), (C.c_uint64 * 3)(*hi), (C.c_uint64 * 3)(*stride),
                            (C.c_void_p * 3)(*[x.ctypes.data for x in inv]), len(fr), fr.ctypes.data, interval)
        i = C.c_size_t()
        self._ck(self._lib.ems_gpu_freq_dump_add(self._h, C.byref(spec), C.byref(i)))
        dims = [(hi[a] - lo[a]) // stride[a] + 1 for a in range(3)]
        self._dumps = getattr(self, "_dumps", {})
        self._dumps[i.value] = (dims, len(fr))
        return i.value

    def add_sampled_freq_dump(self, sampler: "Sampler", freqs, interval: int = 1) -> int:
        """``FreqDump::new(sampler, freqs).interval(interval)`` (src/engine/dump.rs:1420-1700):
        a running DFT on the device of the sampler's quantity at its points."""
        fr = np.ascontiguousarray(freqs, dtype=np.float64)
        z3 = (C.c_uint64 * 3)(0, 0, 0)
        spec = FreqDumpSpec(0, z3, z3, z3, (C.c_void_p * 3)(None, None, None), len(fr), fr.ctypes.data, interval,
                            sampler.table)
        i = C.c_size_t()
        self._ck(self._lib.ems_gpu_freq_dump_add(self._h, C.byref(spec), C.byref(i)))
        self._dumps = getattr(self, "_dumps", {})
        self._dumps[i.value] = (list(sampler.dims), len(fr))
        return i.value

    def add_sampled_time_dump(self, sampler: "Sampler", interval: int = 1) -> int:
        """``TimeDump::new(sampler).schedule(Schedule::Every(interval))`` (src/engine/dump.rs:
        1230-1418): snapshots of the sampler's quantity kept on the device (f64)."""
        z3 = (C.c_uint64 * 3)(0, 0, 0)
        spec = TimeDumpSpec(0, z3, z3, z3, (C.c_void_p * 3)(None, None, None), interval, sampler.table)
        i = C.c_size_t()
        self._ck(self._lib.ems_gpu_time_dump_add(self._h, C.byref(spec), C.byref(i)))
        self._tdumps = getattr(self, "_tdumps", {})
        self._tdumps[i.value] = list(sampler.dims)
        return i.value

    def upml_state(self, op: int, side: int, n: int):
        """(F, v) of the openEMS PML operator ``op``, side 0 E / 1 H."""
        f = np.empty(n, dtype=np.float32)
        v = np.empty(n, dtype=np.float32)
        if n:
            self._ck(self._lib.ems_gpu_upml_state(self._h, op, side, f.ctypes.data, v.ctypes.data, n))
        return f, v

    def add_time_dump(self, field: int, lo, hi, stride=(1, 1, 1), interval: int = 1) -> int:
        """Time-domain snapshots of E (field 0) or H (field 1) over the node
        box lo..hi every ``interval`` states, kept on the device
        (``ems_gpu_time_dump_add``). Returns the dump id."""
        m = self._model
        inv = [m.inv_edge_lengths(a, dual=field == 1) for a in range(3)]
        spec = TimeDumpSpec(field, (C.c_uint64 * 3)(*lo), (C.c_uint64 * 3)(*hi), (C.c_uint64 * 3)(*stride),
                            (C.c_void_p * 3)(*[x.ctypes.data for x in inv]), interval)
        self._inv_keep = getattr(self, "_inv_keep", []) + [inv]
        i = C.c_size_t()
        self._ck(self._lib.ems_gpu_time_dump_add(self._h, C.byref(spec), C.byref(i)))
        self._tdumps = getattr(self, "_tdumps", {})
        self._tdumps[i.value] = [(hi[a] - lo[a]) // stride[a] + 1 for a in range(3)]
        return i.value

    def time_dump(self, dump: int) -> tuple[np.ndarray, np.ndarray]:
        """(states, values): the state m of every snapshot and the values,
        shape (snapshots, nx, ny, nz, 3)."""
        dims = self._tdumps[dump]
        n = C.c_size_t()
        self._ck(self._lib.ems_gpu_time_dump_count(self._h, dump, C.byref(n)))
        pts = int(np.prod(dims))
        vals = np.empty((n.value, pts * 3), dtype=np.float64)
        states = np.empty(n.value, dtype=np.uint64)
        st = C.c_uint64()
        for k in range(n.value):
            self._ck(self._lib.ems_gpu_time_dump_read(self._h, dump, k, vals[k].ctypes.data, pts * 3, C.byref(st)))
            states[k] = st.value
        return states, vals.reshape(n.value, *dims, 3)

    def freq_dump(self, dump: int, k: int) -> np.ndarray:
        """The transform at frequency index k: complex (nx, ny, nz, 3)."""
        dims, _ = self._dumps[dump]
        n = int(np.prod(dims))
        out = np.empty(n * 6, dtype=np.float64)
        self._ck(self._lib.ems_gpu_freq_dump_read(self._h, dump, k, out.ctypes.data, out.size))
        c = out[0::2] + 1j * out[1::2]
        return c.reshape(*dims, 3)

    def autotune(self, cache_path: str) -> None:
        """Schedule autotuning (``ems_gpu_autotune``): cached pick, or timed
        over the next steps ``run`` takes."""
        self._ck(self._lib.ems_gpu_autotune(self._h, os.fsencode(cache_path)))

    @property
    def stream(self) -> int:
        """The engine's cudaStream_t (as an integer address)."""
        p = C.c_void_p()
        self._ck(self._lib.ems_gpu_stream(self._h, C.byref(p)))
        return p.value or 0

    def profile(self, enable: bool = True) -> None:
        self._ck(self._lib.ems_gpu_profile(self._h, 1 if enable else 0))

    def profile_read(self, kernel: int) -> tuple[float, int]:
        """(device ms, launches) of kernel 0 H update, 1 E update, 2 fused step."""
        ms, n = C.c_double(), C.c_uint64()
        self._ck(self._lib.ems_gpu_profile_read(self._h, kernel, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def field(self, field: int, axis: int) -> np.ndarray:
        """``u_component`` (field 0) / ``i_component`` (field 1), shape nodes."""
        out = np.empty(self.nodes, dtype=np.float32)
        self._ck(self._lib.ems_gpu_download_field(self._h, field, axis, out.ctypes.data))
        return out

    def set_field(self, field: int, axis: int, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float32)
        self._ck(self._lib.ems_gpu_upload_field(self._h, field, axis, v.ctypes.data))

    def samples(self, op: int, which: int = 0) -> np.ndarray:
        n = C.c_size_t()
        self._ck(self._lib.ems_gpu_samples(self._h, op, which, None, 0, C.byref(n)))
        out = np.empty(n.value, dtype=np.float64)
        if n.value:
            self._ck(self._lib.ems_gpu_samples(self._h, op, which, out.ctypes.data, n.value, C.byref(n)))
        return out

    def last_sample(self, op: int, which: int = 0) -> float:
        x = C.c_double()
        self._ck(self._lib.ems_gpu_last_sample(self._h, op, which, C.byref(x)))
        return x.value

    def source_amplitude(self, op: int, first: int, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._ck(self._lib.ems_gpu_source_amplitude(self._h, op, first, v.ctypes.data, len(v)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.ems_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Batch:
    """Many built :class:`Model` s stepping together on one device
    (``ems_batch_*``): one launch per kernel kind over all models, one CUDA
    graph per step; a frozen model keeps its state."""

    def __init__(self, models: Sequence[Model], device: int = 0, max_steps: int = 100_000):
        self._lib = gpu_lib()
        self._models = list(models)
        arr = (C.c_void_p * len(self._models))(*[m.desc for m in self._models])
        h = C.c_void_p()
        st = self._lib.ems_batch_create(arr, len(self._models), device, max_steps, C.byref(h))
        if st != 0:
            raise EngineError(st, "ems_batch_create failed")
        self._h = h
        self.n = len(self._models)

    def _ck(self, st: int) -> None:
        if st != 0:
            raise EngineError(st, self._lib.ems_batch_last_error(self._h).decode())

    def run(self, n: int) -> None:
        self._ck(self._lib.ems_batch_run(self._h, n))

    def step_with_energy(self) -> np.ndarray:
        w = np.zeros(self.n, dtype=np.float64)
        self._ck(self._lib.ems_batch_step_with_energy(self._h, w.ctypes.data))
        return w

    def set_active(self, model: int, active: bool) -> None:
        self._ck(self._lib.ems_batch_set_active(self._h, model, 1 if active else 0))

    def autotune(self, cache_path: str) -> None:
        """Persistent-grid autotuning (``ems_batch_autotune``)."""
        self._ck(self._lib.ems_batch_autotune(self._h, os.fsencode(cache_path)))

    def timestep(self, model: int) -> int:
        n = C.c_uint64()
        self._ck(self._lib.ems_batch_timestep(self._h, model, C.byref(n)))
        return n.value

    def samples(self, model: int, op: int, which: int = 0) -> np.ndarray:
        n = C.c_size_t()
        self._ck(self._lib.ems_batch_samples(self._h, model, op, which, None, 0, C.byref(n)))
        out = np.empty(n.value, dtype=np.float64)
        if n.value:
            self._ck(self._lib.ems_batch_samples(self._h, model, op, which, out.ctypes.data, n.value, C.byref(n)))
        return out

    def field(self, model: int, field: int, axis: int) -> np.ndarray:
        out = np.empty(self._models[model].nodes, dtype=np.float32)
        self._ck(self._lib.ems_batch_download_field(self._h, model, field, axis, out.ctypes.data))
        return out

    @property
    def stream(self) -> int:
        p = C.c_void_p()
        self._ck(self._lib.ems_batch_stream(self._h, C.byref(p)))
        return p.value or 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.ems_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def run_until(stepper, limits: RunLimits) -> RunOutcome:
    """``Engine::run_until`` (src/engine/run.rs:221-540) over any object with
    ``run(n)`` and ``step_with_energy()``, driven by the host's run loop."""
    lib = host_lib()
    err: list[BaseException] = []

    @C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64)
    def _run(_ctx, n):
        try:
            stepper.run(n)
            return 0
        except BaseException as e:  # surfaced below
            err.append(e)
            return 1

    @C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double))
    def _swe(_ctx, w):
        try:
            w[0] = stepper.step_with_energy()
            return 0
        except EngineError as e:
            if e.status == ERR_DIVERGED:  # an outcome of the run (Diverged), not an error
                w[0] = float("nan")
                return ERR_DIVERGED
            err.append(e)
            return 1
        except BaseException as e:
            err.append(e)
            return 1

    s = Stepper(None, _run, _swe)
    out = RunOutcome()
    lib.ems_drive(C.byref(s), C.byref(limits), C.byref(out))
    if err:
        raise err[0]
    return out


def run_until_batch(batch, limits: Sequence[RunLimits]) -> list[RunOutcome]:
    """The run loop over a batch (``ems_batch_drive``): every model gets the
    outcome ``run_until`` would give it alone; a model that stops is frozen.
    ``batch`` has ``n``, ``run(n)``, ``step_with_energy()`` (one value per
    model) and ``set_active(model, active)``."""
    lib = host_lib()
    err: list[BaseException] = []
    n = batch.n

    @C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64)
    def _run(_ctx, k):
        try:
            batch.run(k)
            return 0
        except BaseException as e:
            err.append(e)
            return 1

    @C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double))
    def _swe(_ctx, w):
        try:
            v = batch.step_with_energy()
            for q in range(n):
                w[q] = float(v[q])
            return 0
        except BaseException as e:
            err.append(e)
            return 1

    @C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_size_t, C.c_int)
    def _act(_ctx, m, a):
        try:
            batch.set_active(m, bool(a))
            return 0
        except BaseException as e:
            err.append(e)
            return 1

    s = BatchStepper(None, n, _run, _swe, _act)
    lims = (RunLimits * n)(*limits)
    outs = (RunOutcome * n)()
    st = lib.ems_batch_drive(C.byref(s), lims, outs)
    if err:
        raise err[0]
    if st != 0:
        raise ValueError("ems_batch_drive: invalid limits (check intervals differ?)")
    return list(outs)


def energy_decay_limits(max_steps: int, db: float, dt: float, excitation_end: float | None = None,
                        interval: int = 50) -> RunLimits:
    """``RunLimits::new(max).end_criteria(EndCriteria::energy_decay_db(db)).excitation_end(end)``."""
    return RunLimits(max_steps, 1, 10.0 ** (db / 10.0), interval, 1 if excitation_end is not None else 0,
                     excitation_end or 0.0, dt)


DUMP_E, DUMP_H, DUMP_J, DUMP_ROTH, DUMP_D, DUMP_B = 0, 1, 2, 3, 4, 5
NODES, CELL_CENTERS, NATIVE = 0, 1, 2
DUMP_NAMES = ("E", "H", "J", "RotH", "D", "B")


class Sampler:
    """``FieldSampler`` (src/engine/dump.rs:487-940): ``quantity`` (DUMP_E … DUMP_B)
    converted to field units and interpolated at the sample points of the node box between
    corners ``a`` and ``b`` (inclusive, any order) with ``stride``, at ``position`` NODES,
    CELL_CENTERS or NATIVE; with ``indices`` (three increasing lists) the explicit points
    and openEMS's rules (``FieldSampler::openems``). The table lives as long as this object."""

    def __init__(self, model: "Model", quantity: int, position: int = NODES, a: Sequence[int] | None = None,
                 b: Sequence[int] | None = None, stride: Sequence[int] = (1, 1, 1),
                 indices: Sequence[Sequence[int]] | None = None):
        self._lib = host_lib()
        self._model = model
        self.quantity, self.position = quantity, position
        if indices is not None:
            arrs = [np.ascontiguousarray(v, dtype=np.uint64) for v in indices]
            ptrs = (C.c_void_p * 3)(*[x.ctypes.data for x in arrs])
            ns = (C.c_size_t * 3)(*[len(x) for x in arrs])
            h = self._lib.ems_sampler_new_indices(model._p, quantity, position, ptrs, ns)
        else:
            n = model.nodes
            a = [0, 0, 0] if a is None else list(a)
            b = [x - 1 for x in n] if b is None else list(b)
            h = self._lib.ems_sampler_new(model._p, quantity, position, _u64(a), _u64(b), _u64(stride))
        if not h:
            raise ValueError(f"sampler: {self._lib.ems_model_error(model._p).decode()}")
        self._h = h
        self.table = self._lib.ems_sampler_table(h)
        self.coords = []
        for ax in range(3):
            cnt = C.c_size_t()
            ptr = self._lib.ems_sampler_coords(h, ax, C.byref(cnt))
            self.coords.append(np.ctypeslib.as_array((C.c_double * cnt.value).from_address(ptr)).copy())
        self.dims = tuple(len(c) for c in self.coords)

    @property
    def name(self) -> str:
        return DUMP_NAMES[self.quantity]

    @property
    def from_currents(self) -> bool:
        return self.quantity in (DUMP_H, DUMP_B, DUMP_ROTH)

    def __len__(self) -> int:
        return int(np.prod(self.dims))

    def time(self, state: int, dt: float) -> float:
        """``FieldSampler::time`` with ``DumpTiming::State`` (dump.rs:786-812)."""
        return (state - 0.5 if self.from_currents else float(state)) * dt

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.ems_sampler_free(h)
            self._h = None


def sheet_rect_edges(normal: int, plane: int, start: Sequence[int], stop: Sequence[int], sigma: float,
                     t: float) -> list[tuple]:
    """The edges ``ConductingSheet::add_rect`` pushes (src/engine/sheet.rs:573-603): for
    (d, o) in ((next, prev), (prev, next)) of the normal, d from start to stop − 1 and o
    from start to stop, on node plane ``plane``."""
    p, q = (normal + 1) % 3, (normal + 2) % 3
    out = []
    for d, o in ((p, q), (q, p)):
        for a in range(start[d], stop[d]):
            for b in range(start[o], stop[o] + 1):
                node = [0, 0, 0]
                node[normal], node[d], node[o] = plane, a, b
                out.append((d, tuple(node), normal, sigma, t))
    return out


def skin_depth(sigma: float, f: float) -> float:
    """``skin_depth`` (src/engine/sheet.rs:237-239): √(2/(ω·μ0·σ))."""
    return math.sqrt(2.0 / (2.0 * math.pi * f * mu0() * sigma))


def layer_profile(sigma: float, thickness: float, f_max: float) -> np.ndarray:
    """``layer_profile`` (src/engine/sheet.rs:244-271), from the host library."""
    L = host_lib()
    n = L.ems_sheet_layer_profile(sigma, thickness, f_max, None, 0)
    out = np.zeros(max(n, 1))
    L.ems_sheet_layer_profile(sigma, thickness, f_max, out.ctypes.data, len(out))
    return out[:n]


def _coth_csch(x: complex) -> tuple[complex, complex]:
    e1 = cmath.exp(-x)
    e2 = e1 * e1
    den = 1.0 - e2
    return (1.0 + e2) / den, e1 * 2.0 / den


def _csqrt(z: complex) -> complex:
    r, a = cmath.polar(z)
    return cmath.rect(math.sqrt(r), 0.5 * a)


def slab_impedance(sigma: float, t: float, f: float) -> tuple[complex, complex]:
    """``slab_impedance`` (src/engine/sheet.rs:288-298): [Z11, Z12] per square of the exact
    slab, Z_c·coth(γt) and Z_c·csch(γt)."""
    w = 2.0 * math.pi * f
    y = complex(sigma, w * eps0())
    jwm = complex(0.0, w * mu0())
    gamma = _csqrt(jwm * y)
    zc = _csqrt(jwm / y)
    coth, csch = _coth_csch(gamma * t)
    return zc * coth, zc * csch


def _z_to_abcd(z11: complex, z12: complex) -> list[complex]:
    a = z11 / z12
    return [a, (z11 * z11 - z12 * z12) / z12, 1.0 / z12, a]


def slab_abcd(sigma: float, t: float, f: float) -> list[complex]:
    """``slab_abcd`` (src/engine/sheet.rs:300-303): the exact slab's chain matrix."""
    return _z_to_abcd(*slab_impedance(sigma, t, f))


def model_abcd(sigma: float, t: float, f_max: float, f: float) -> list[complex]:
    """``model_abcd`` (src/engine/sheet.rs:313-345): the chain matrix of the ladder the
    operator integrates (continuous time), shunt half layers at the ends."""
    w = 2.0 * math.pi * f
    dz = layer_profile(sigma, t, f_max)

    def mul(m, n):
        return [m[0] * n[0] + m[1] * n[2], m[0] * n[1] + m[1] * n[3],
                m[2] * n[0] + m[3] * n[2], m[2] * n[1] + m[3] * n[3]]

    def shunt(v):
        return [1.0 + 0j, 0j, complex(sigma * v, w * eps0() * v), 1.0 + 0j]

    def series(ln):
        return [1.0 + 0j, complex(0.0, w * mu0() * ln), 0j, 1.0 + 0j]

    m = shunt(0.5 * dz[0])
    for k, d in enumerate(dz):
        m = mul(m, series(d))
        m = mul(m, shunt(0.5 * (d + (dz[k + 1] if k + 1 < len(dz) else 0.0))))
    return m


def dft(t0: float, dt: float, x: np.ndarray, freqs: Sequence[float]) -> np.ndarray:
    """``post::dft`` (src/post/dft.rs:218): Σ x(t0+n·dt)·e^{-j2πf·t_n}·dt."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    f = np.ascontiguousarray(freqs, dtype=np.float64)
    re = np.empty(len(f))
    im = np.empty(len(f))
    host_lib().ems_dft(t0, dt, x.ctypes.data, len(x), f.ctypes.data, len(f), re.ctypes.data, im.ctypes.data)
    return re + 1j * im


class PortResult:
    """``PortResult`` (src/post/port.rs:60-230): a port's V(f), I(f) and its
    reference impedance, with the power waves, S11, Z_in and powers."""

    def __init__(self, freqs: Sequence[float], v: np.ndarray, i: np.ndarray, z_ref: complex):
        self.freqs = np.asarray(freqs, dtype=np.float64)
        self.v = np.asarray(v, dtype=complex)
        self.i = np.asarray(i, dtype=complex)
        self.z_ref = complex(z_ref)

    @classmethod
    def of_port(cls, v: np.ndarray, i: np.ndarray, dt: float, freqs: Sequence[float], z_ref: complex):
        """``LumpedPort::analyze_with`` (src/engine/port.rs:202-215): DFTs of V
        sampled at (n+1)·dt and I at (n+½)·dt."""
        return cls(freqs, dft(dt, dt, v, freqs), dft(0.5 * dt, dt, i, freqs), z_ref)

    def a(self) -> np.ndarray:
        return (self.v + self.z_ref * self.i) * (0.5 / math.sqrt(self.z_ref.real))

    def b(self) -> np.ndarray:
        return (self.v - self.z_ref.conjugate() * self.i) * (0.5 / math.sqrt(self.z_ref.real))

    def z_in(self) -> np.ndarray:
        return self.v / self.i

    def s11(self) -> np.ndarray:
        return s_param(self, self)

    def incident_power(self) -> np.ndarray:
        return 0.5 * np.abs(self.a()) ** 2

    def reflected_power(self) -> np.ndarray:
        return 0.5 * np.abs(self.b()) ** 2

    def accepted_power(self) -> np.ndarray:
        return 0.5 * (self.v.real * self.i.real + self.v.imag * self.i.imag)


def s_param(out: PortResult, inc: PortResult) -> np.ndarray:
    """``s_param`` (src/post/port.rs:236-242): S_oi = b_o / a_i."""
    assert np.array_equal(out.freqs, inc.freqs), "port results at different frequencies"
    return out.b() / inc.a()


def port_result(v: np.ndarray, i: np.ndarray, dt: float, freqs: Sequence[float], z_ref: float = 50.0):
    """``LumpedPort::analyze`` (src/engine/port.rs:191-205) → (Z_in, S11) per
    frequency (src/post/port.rs:202-209): V at (n+1)dt, I at (n+½)dt."""
    V = dft(dt, dt, v, freqs)
    I = dft(0.5 * dt, dt, i, freqs)
    z_in = V / I
    a = (V + z_ref * I) / (2.0 * np.sqrt(z_ref))
    b = (V - np.conj(z_ref) * I) / (2.0 * np.sqrt(z_ref))
    return z_in, b / a
