"""Python host binding of libfullmag_fdm.so.0 over its C ABI.

Mirrors the reference's safe Rust wrapper ``NativeFdmBackend``
(crates/fullmag-runner/src/native_fdm.rs:90-704): a plan is turned into a
``fullmag_fdm_plan_desc``, the handle is created and its deferred error
checked, then ``step`` / ``copy_m`` / ``copy_field`` / previews / snapshots /
uploads go straight to the library.  Errors raise ``RunError`` with the
library's ``last_error`` text, like the Rust ``RunError`` mapping
(native_fdm.rs:696-704).

There is no CPU fallback: loading fails loudly when the library or a CUDA
device is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

import numpy as np

from . import build as _build

MU0 = 4.0 * np.pi * 1e-7

OK, ERR_INVALID, ERR_CUDA, ERR_INTERNAL = 0, -1, -2, -3
PRECISION_SINGLE, PRECISION_DOUBLE = 1, 2
HEUN, DP45, ABM3, RK4, RK23 = 1, 2, 3, 4, 5
BOUNDARY_NONE, BOUNDARY_VOLUME, BOUNDARY_FULL = 0, 1, 2
OBS_M, OBS_H_EX, OBS_H_DEMAG, OBS_H_EXT, OBS_H_EFF = 1, 2, 3, 4, 5
SNAP_F32, SNAP_F64 = 1, 2
DEMAG_FROM_PLAN, DEMAG_NEWELL = 0, 1
MAX_EXCHANGE_REGIONS = 256

_dp = C.POINTER(C.c_double)


class GridDesc(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double)]


class MaterialDesc(C.Structure):
    _fields_ = [("saturation_magnetisation", C.c_double), ("exchange_stiffness", C.c_double),
                ("damping", C.c_double), ("gyromagnetic_ratio", C.c_double)]


class PlanDesc(C.Structure):
    _fields_ = [
        ("grid", GridDesc), ("material", MaterialDesc),
        ("precision", C.c_int), ("integrator", C.c_int),
        ("disable_precession", C.c_int), ("enable_exchange", C.c_int),
        ("enable_demag", C.c_int), ("has_external_field", C.c_int),
        ("external_field_am", C.c_double * 3),
        ("demag_kernel_xx_spectrum", _dp), ("demag_kernel_yy_spectrum", _dp),
        ("demag_kernel_zz_spectrum", _dp), ("demag_kernel_xy_spectrum", _dp),
        ("demag_kernel_xz_spectrum", _dp), ("demag_kernel_yz_spectrum", _dp),
        ("demag_kernel_spectrum_len", C.c_uint64),
        ("active_mask", C.POINTER(C.c_uint8)), ("active_mask_len", C.c_uint64),
        ("region_mask", C.POINTER(C.c_uint32)), ("region_mask_len", C.c_uint64),
        ("exchange_lut", _dp), ("exchange_lut_len", C.c_uint64),
        ("boundary_correction", C.c_int), ("boundary_phi_floor", C.c_double),
        ("boundary_delta_min", C.c_double),
        ("volume_fraction", _dp), ("volume_fraction_len", C.c_uint64),
        ("face_link_xp", _dp), ("face_link_xm", _dp), ("face_link_yp", _dp),
        ("face_link_ym", _dp), ("face_link_zp", _dp), ("face_link_zm", _dp),
        ("delta_xp", _dp), ("delta_xm", _dp), ("delta_yp", _dp),
        ("delta_ym", _dp), ("delta_zp", _dp), ("delta_zm", _dp),
        ("has_demag_boundary_corr", C.c_int),
        ("demag_corr_target_idx", C.POINTER(C.c_int32)),
        ("demag_corr_source_idx", C.POINTER(C.c_int32)),
        ("demag_corr_tensor", _dp),
        ("demag_corr_target_count", C.c_uint32), ("demag_corr_stencil_size", C.c_uint32),
        ("initial_magnetization_xyz", _dp), ("initial_magnetization_len", C.c_uint64),
        ("adaptive_max_error", C.c_double), ("adaptive_dt_min", C.c_double),
        ("adaptive_dt_max", C.c_double), ("adaptive_headroom", C.c_double),
    ]


class StepStats(C.Structure):
    _fields_ = [("step", C.c_uint64), ("time_seconds", C.c_double), ("dt_seconds", C.c_double),
                ("exchange_energy_joules", C.c_double), ("demag_energy_joules", C.c_double),
                ("external_energy_joules", C.c_double), ("total_energy_joules", C.c_double),
                ("max_effective_field_amplitude", C.c_double),
                ("max_demag_field_amplitude", C.c_double), ("max_rhs_amplitude", C.c_double),
                ("suggested_next_dt", C.c_double), ("wall_time_ns", C.c_uint64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class DeviceInfo(C.Structure):
    _fields_ = [("name", C.c_char * 128), ("compute_capability_major", C.c_int),
                ("compute_capability_minor", C.c_int), ("driver_version", C.c_int),
                ("runtime_version", C.c_int)]


class SnapshotDesc(C.Structure):
    _fields_ = [("cell_count", C.c_uint64), ("component_count", C.c_uint32),
                ("scalar_bytes", C.c_uint32), ("scalar_type", C.c_int)]


class PlanExt(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("ms_map", _dp), ("ms_map_len", C.c_uint64),
                ("ac_field_am", C.c_double * 3), ("ac_frequency_hz", C.c_double),
                ("demag_source", C.c_int)]


# Every function declared in include/fullmag_fdm.h and include/fullmag_fdm_ext.h.
ABI_FUNCTIONS = (
    "fullmag_fdm_is_available", "fullmag_fdm_backend_create", "fullmag_fdm_backend_step",
    "fullmag_fdm_backend_copy_field_f64", "fullmag_fdm_backend_copy_field_f32",
    "fullmag_fdm_backend_copy_field_preview_f64", "fullmag_fdm_backend_copy_field_preview_f32",
    "fullmag_fdm_backend_begin_field_snapshot", "fullmag_fdm_field_snapshot_wait",
    "fullmag_fdm_field_snapshot_destroy", "fullmag_fdm_backend_upload_magnetization_f64",
    "fullmag_fdm_backend_upload_magnetization_f32", "fullmag_fdm_backend_refresh_observables",
    "fullmag_fdm_backend_get_device_info", "fullmag_fdm_backend_last_error",
    "fullmag_fdm_backend_destroy",
)
EXT_FUNCTIONS = (
    "fullmag_fdm_backend_create_ext", "fullmag_fdm_backend_step_n",
    "fullmag_fdm_backend_set_profiling", "fullmag_fdm_backend_profile_count",
    "fullmag_fdm_backend_profile_entry", "fullmag_fdm_backend_profile_reset",
    "fullmag_fdm_backend_memory_info", "fullmag_fdm_newell_spectra",
    "fullmag_fdm_backend_get_stream", "fullmag_fdm_random_unit_vectors",
    "fullmag_fdm_adjoint_forward", "fullmag_fdm_adjoint_backward",
    "fullmag_fdm_batch_create", "fullmag_fdm_batch_step_n", "fullmag_fdm_batch_copy_m",
    "fullmag_fdm_batch_tuning", "fullmag_fdm_batch_last_error", "fullmag_fdm_batch_destroy",
    "fullmag_fdm_batch_get_stream", "fullmag_fdm_batch_profile_step",
)

class BatchProblem(C.Structure):
    """fullmag_fdm_batch_problem (include/fullmag_fdm_ext.h)."""
    _fields_ = [
        ("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("saturation_magnetisation", C.c_double), ("exchange_stiffness", C.c_double),
        ("damping", C.c_double), ("gyromagnetic_ratio", C.c_double),
        ("external_field_am", C.c_double * 3),
        ("initial_magnetization_xyz", _dp),
    ]


_lib = None


def library_path() -> str:
    return _build.LIB


def load_library(build_if_missing: bool = True):
    """Load libfullmag_fdm.so.0 from the package (build it with nvcc if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        if not build_if_missing:
            raise RuntimeError(f"{path} is missing; run fullmag_b200/build.py")
        _build.build()
    L = C.CDLL(path)
    vp = C.c_void_p
    L.fullmag_fdm_is_available.restype = C.c_int
    L.fullmag_fdm_backend_create.restype = vp
    L.fullmag_fdm_backend_create.argtypes = [C.POINTER(PlanDesc)]
    L.fullmag_fdm_backend_create_ext.restype = vp
    L.fullmag_fdm_backend_create_ext.argtypes = [C.POINTER(PlanDesc), C.POINTER(PlanExt)]
    L.fullmag_fdm_backend_step.argtypes = [vp, C.c_double, C.POINTER(StepStats)]
    L.fullmag_fdm_backend_step_n.argtypes = [vp, C.c_double, C.c_uint32, C.POINTER(StepStats)]
    L.fullmag_fdm_backend_copy_field_f64.argtypes = [vp, C.c_int, _dp, C.c_uint64]
    L.fullmag_fdm_backend_copy_field_f32.argtypes = [vp, C.c_int, C.POINTER(C.c_float), C.c_uint64]
    L.fullmag_fdm_backend_copy_field_preview_f64.argtypes = [vp, C.c_int] + [C.c_uint32] * 5 + [_dp, C.c_uint64]
    L.fullmag_fdm_backend_copy_field_preview_f32.argtypes = [vp, C.c_int] + [C.c_uint32] * 5 + [C.POINTER(C.c_float), C.c_uint64]
    L.fullmag_fdm_backend_begin_field_snapshot.restype = vp
    L.fullmag_fdm_backend_begin_field_snapshot.argtypes = [vp, C.c_int]
    L.fullmag_fdm_field_snapshot_wait.argtypes = [vp, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64), C.POINTER(SnapshotDesc)]
    L.fullmag_fdm_field_snapshot_destroy.argtypes = [vp]
    L.fullmag_fdm_field_snapshot_destroy.restype = None
    L.fullmag_fdm_backend_upload_magnetization_f64.argtypes = [vp, _dp, C.c_uint64]
    L.fullmag_fdm_backend_upload_magnetization_f32.argtypes = [vp, C.POINTER(C.c_float), C.c_uint64]
    L.fullmag_fdm_backend_refresh_observables.argtypes = [vp]
    L.fullmag_fdm_backend_get_device_info.argtypes = [vp, C.POINTER(DeviceInfo)]
    L.fullmag_fdm_backend_last_error.restype = C.c_char_p
    L.fullmag_fdm_backend_last_error.argtypes = [vp]
    L.fullmag_fdm_backend_destroy.argtypes = [vp]
    L.fullmag_fdm_backend_destroy.restype = None
    L.fullmag_fdm_backend_set_profiling.argtypes = [vp, C.c_int]
    L.fullmag_fdm_backend_profile_count.argtypes = [vp]
    L.fullmag_fdm_backend_profile_entry.argtypes = [vp, C.c_int, C.POINTER(C.c_char_p), _dp, C.POINTER(C.c_uint64)]
    L.fullmag_fdm_backend_profile_reset.argtypes = [vp]
    L.fullmag_fdm_backend_profile_reset.restype = None
    L.fullmag_fdm_backend_memory_info.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]
    L.fullmag_fdm_newell_spectra.argtypes = [C.c_uint32] * 3 + [C.c_double] * 3 + [C.c_int] + [_dp] * 6
    L.fullmag_fdm_backend_get_stream.argtypes = [vp, C.POINTER(C.c_void_p)]
    L.fullmag_fdm_random_unit_vectors.argtypes = [C.c_uint64, C.c_uint64, _dp]
    L.fullmag_fdm_random_unit_vectors.restype = None
    L.fullmag_fdm_adjoint_forward.argtypes = [vp, C.c_double, C.c_uint32, C.c_uint32, C.POINTER(StepStats)]
    L.fullmag_fdm_adjoint_backward.argtypes = [vp, _dp, C.c_uint64, _dp, _dp, _dp, _dp]
    L.fullmag_fdm_batch_create.restype = vp
    L.fullmag_fdm_batch_create.argtypes = [C.POINTER(BatchProblem), C.c_uint32, C.c_int]
    L.fullmag_fdm_batch_step_n.argtypes = [vp, C.c_double, C.c_uint32]
    L.fullmag_fdm_batch_copy_m.argtypes = [vp, C.c_uint32, _dp, C.c_uint64]
    L.fullmag_fdm_batch_tuning.argtypes = [vp, C.POINTER(C.c_int32), C.c_uint32]
    L.fullmag_fdm_batch_last_error.restype = C.c_char_p
    L.fullmag_fdm_batch_last_error.argtypes = [vp]
    L.fullmag_fdm_batch_destroy.argtypes = [vp]
    L.fullmag_fdm_batch_get_stream.argtypes = [vp, C.POINTER(C.c_void_p)]
    L.fullmag_fdm_batch_profile_step.argtypes = [vp, C.c_double, C.POINTER(C.c_float), C.c_uint32]
    L.fullmag_fdm_batch_destroy.restype = None
    _lib = L
    return L


def is_available() -> bool:
    return bool(load_library().fullmag_fdm_is_available())


class RunError(RuntimeError):
    pass


def random_unit_vectors(seed: int, count: int) -> np.ndarray:
    """Seeded m0 as the reference planner draws it (fullmag-plan/src/lib.rs:1928-1957)."""
    out = np.zeros(3 * int(count))
    load_library().fullmag_fdm_random_unit_vectors(int(seed), int(count), out.ctypes.data_as(_dp))
    return out


def newell_spectra(nx: int, ny: int, nz: int, dx: float, dy: float, dz: float,
                   thin_film_2d: bool = False):
    """FP64 Newell spectra in the reference's interleaved complex layout (host code)."""
    pz = 1 if (thin_film_2d and nz == 1) else 2 * nz
    p = 4 * nx * ny * pz
    outs = [np.zeros(2 * p) for _ in range(6)]
    rc = load_library().fullmag_fdm_newell_spectra(nx, ny, nz, dx, dy, dz, int(thin_film_2d),
                                                   *[o.ctypes.data_as(_dp) for o in outs])
    if rc != OK:
        raise RunError(f"fullmag_fdm_newell_spectra failed ({rc})")
    return outs


@dataclass
class FdmPlan:
    """The FdmPlanIR fields the reference runner maps into the plan descriptor
    (crates/fullmag-runner/src/native_fdm.rs:90-346)."""
    cells: Tuple[int, int, int]
    cell_size: Tuple[float, float, float]
    initial_magnetization: np.ndarray           # AoS [3N] or (N, 3)
    saturation_magnetisation: float = 8.0e5
    exchange_stiffness: float = 1.3e-11
    damping: float = 0.02
    gyromagnetic_ratio: float = 2.211e5
    precision: int = PRECISION_DOUBLE
    integrator: int = HEUN
    pure_damping: bool = False
    enable_exchange: bool = True
    enable_demag: bool = True
    external_field: Optional[Sequence[float]] = None   # A/m
    active_mask: Optional[np.ndarray] = None
    region_mask: Optional[np.ndarray] = None
    exchange_lut: Optional[np.ndarray] = None
    demag_spectra: Optional[Sequence[np.ndarray]] = None  # 6 interleaved arrays
    adaptive: Optional[Tuple[float, float, float, float]] = None  # max_error, dt_min, dt_max, headroom
    # extension block
    ms_map: Optional[np.ndarray] = None
    ac_field: Optional[Sequence[float]] = None
    ac_frequency_hz: float = 0.0
    demag_source: int = DEMAG_FROM_PLAN
    # boundary tiers (fullmag_fdm.h:151-187): BOUNDARY_NONE / _VOLUME (T0) / _FULL (T1);
    # per-cell arrays of N doubles, directions in the order xp, xm, yp, ym, zp, zm
    boundary_correction: int = 0
    boundary_phi_floor: float = 0.0
    boundary_delta_min: float = 0.0
    volume_fraction: Optional[np.ndarray] = None
    face_links: Optional[Sequence[np.ndarray]] = None
    deltas: Optional[Sequence[np.ndarray]] = None
    # sparse demag correction: targets [T], sources [T, S], tensors [T, S, 6]
    demag_corr: Optional[Tuple[np.ndarray, np.ndarray, np.ndarray]] = None
    _keep: list = field(default_factory=list, repr=False)

    @property
    def cell_count(self) -> int:
        return int(self.cells[0] * self.cells[1] * self.cells[2])

    def to_desc(self) -> PlanDesc:
        d = PlanDesc()
        keep = self._keep = []
        d.grid.nx, d.grid.ny, d.grid.nz = (int(c) for c in self.cells)
        d.grid.dx, d.grid.dy, d.grid.dz = (float(c) for c in self.cell_size)
        d.material.saturation_magnetisation = self.saturation_magnetisation
        d.material.exchange_stiffness = self.exchange_stiffness
        d.material.damping = self.damping
        d.material.gyromagnetic_ratio = self.gyromagnetic_ratio
        d.precision = self.precision
        d.integrator = self.integrator
        d.disable_precession = int(self.pure_damping)
        d.enable_exchange = int(self.enable_exchange)
        d.enable_demag = int(self.enable_demag)
        d.has_external_field = int(self.external_field is not None)
        for i, v in enumerate(self.external_field or (0.0, 0.0, 0.0)):
            d.external_field_am[i] = float(v)
        if self.demag_spectra is not None:
            names = ("xx", "yy", "zz", "xy", "xz", "yz")
            for nm, arr in zip(names, self.demag_spectra):
                a = np.ascontiguousarray(arr, dtype=np.float64)
                keep.append(a)
                setattr(d, f"demag_kernel_{nm}_spectrum", a.ctypes.data_as(_dp))
            d.demag_kernel_spectrum_len = int(np.asarray(self.demag_spectra[0]).size)
        if self.active_mask is not None:
            a = np.ascontiguousarray(self.active_mask, dtype=np.uint8)
            keep.append(a)
            d.active_mask = a.ctypes.data_as(C.POINTER(C.c_uint8))
            d.active_mask_len = a.size
        if self.region_mask is not None:
            a = np.ascontiguousarray(self.region_mask, dtype=np.uint32)
            keep.append(a)
            d.region_mask = a.ctypes.data_as(C.POINTER(C.c_uint32))
            d.region_mask_len = a.size
        if self.exchange_lut is not None:
            a = np.ascontiguousarray(self.exchange_lut, dtype=np.float64)
            keep.append(a)
            d.exchange_lut = a.ctypes.data_as(_dp)
            d.exchange_lut_len = a.size
        m0 = np.ascontiguousarray(self.initial_magnetization, dtype=np.float64).reshape(-1)
        keep.append(m0)
        d.initial_magnetization_xyz = m0.ctypes.data_as(_dp)
        d.initial_magnetization_len = m0.size
        if self.adaptive is not None:
            (d.adaptive_max_error, d.adaptive_dt_min, d.adaptive_dt_max,
             d.adaptive_headroom) = (float(v) for v in self.adaptive)
        d.boundary_correction = int(self.boundary_correction)
        d.boundary_phi_floor = float(self.boundary_phi_floor)
        d.boundary_delta_min = float(self.boundary_delta_min)

        def dptr(arr):
            a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
            keep.append(a)
            return a.ctypes.data_as(_dp), a.size

        if self.volume_fraction is not None:
            d.volume_fraction, d.volume_fraction_len = dptr(self.volume_fraction)
        dirs = ("xp", "xm", "yp", "ym", "zp", "zm")
        if self.face_links is not None:
            for nm, arr in zip(dirs, self.face_links):
                setattr(d, f"face_link_{nm}", dptr(arr)[0])
        if self.deltas is not None:
            for nm, arr in zip(dirs, self.deltas):
                setattr(d, f"delta_{nm}", dptr(arr)[0])
        if self.demag_corr is not None:
            tgt, src, ten = self.demag_corr
            t = np.ascontiguousarray(tgt, dtype=np.int32).reshape(-1)
            sr = np.ascontiguousarray(src, dtype=np.int32).reshape(-1)
            keep.extend([t, sr])
            d.has_demag_boundary_corr = 1
            d.demag_corr_target_idx = t.ctypes.data_as(C.POINTER(C.c_int32))
            d.demag_corr_source_idx = sr.ctypes.data_as(C.POINTER(C.c_int32))
            d.demag_corr_tensor = dptr(ten)[0]
            d.demag_corr_target_count = t.size
            d.demag_corr_stencil_size = sr.size // max(t.size, 1)
        return d

    def to_ext(self) -> Optional[PlanExt]:
        if self.ms_map is None and self.ac_field is None and self.demag_source == DEMAG_FROM_PLAN:
            return None
        e = PlanExt()
        e.struct_size = C.sizeof(PlanExt)
        if self.ms_map is not None:
            a = np.ascontiguousarray(self.ms_map, dtype=np.float64)
            self._keep.append(a)
            e.ms_map = a.ctypes.data_as(_dp)
            e.ms_map_len = a.size
        for i, v in enumerate(self.ac_field or (0.0, 0.0, 0.0)):
            e.ac_field_am[i] = float(v)
        e.ac_frequency_hz = float(self.ac_frequency_hz)
        e.demag_source = int(self.demag_source)
        return e


class NativeFdmBackend:
    """RAII handle over fullmag_fdm_backend (native_fdm.rs:90-704)."""

    def __init__(self, plan: FdmPlan):
        self._lib = load_library()
        self.plan = plan
        self.n = plan.cell_count
        self.precision = plan.precision
        desc = plan.to_desc()
        ext = plan.to_ext()
        self._desc = desc
        if ext is None:
            h = self._lib.fullmag_fdm_backend_create(C.byref(desc))
        else:
            self._ext = ext
            h = self._lib.fullmag_fdm_backend_create_ext(C.byref(desc), C.byref(ext))
        if not h:
            raise RunError("CUDA FDM backend_create returned null")
        err = self._lib.fullmag_fdm_backend_last_error(h)
        if err is not None:
            self._lib.fullmag_fdm_backend_destroy(h)
            raise RunError(err.decode())
        self._h = h
        self._st = StepStats()
        self._st_ref = C.byref(self._st)

    # -- lifecycle --
    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h:
            self._lib.fullmag_fdm_backend_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, rc: int, what: str) -> None:
        if rc != OK:
            err = self._lib.fullmag_fdm_backend_last_error(self._h)
            raise RunError(f"{what} failed ({rc}): {err.decode() if err else 'unknown error'}")

    # -- stepping --
    def step(self, dt: float) -> dict:
        st = self._st  # one statistics buffer per backend, filled by every call
        self._check(self._lib.fullmag_fdm_backend_step(self._h, dt, self._st_ref), "step")
        return st.as_dict()

    def step_n(self, dt: float, n: int) -> dict:
        st = StepStats()
        self._check(self._lib.fullmag_fdm_backend_step_n(self._h, dt, n, C.byref(st)), "step_n")
        return st.as_dict()

    # -- adjoint of a Heun trajectory (fullmag_fdm_ext.h) --
    def adjoint_forward(self, dt: float, n: int, checkpoint_every: int = 0) -> dict:
        """n Heun steps from the current state, keeping device checkpoints
        every `checkpoint_every` steps (0: ceil(sqrt(n)))."""
        st = StepStats()
        self._check(self._lib.fullmag_fdm_adjoint_forward(self._h, dt, n, checkpoint_every, C.byref(st)),
                    "adjoint_forward")
        return st.as_dict()

    def adjoint_backward(self, dl_dm: np.ndarray) -> dict:
        """dL/dm at the final state (AoS 3N) -> dL/dMs per cell, dL/dH_ext (3,),
        dL/dH_ac (3,) in A/m, and dL/dm0 (AoS 3N)."""
        g = np.ascontiguousarray(dl_dm, dtype=np.float64).reshape(-1)
        gms = np.zeros(self.n)
        ge = np.zeros(3)
        ga = np.zeros(3)
        g0 = np.zeros(3 * self.n)
        self._check(self._lib.fullmag_fdm_adjoint_backward(
            self._h, g.ctypes.data_as(_dp), g.size, gms.ctypes.data_as(_dp), ge.ctypes.data_as(_dp),
            ga.ctypes.data_as(_dp), g0.ctypes.data_as(_dp)), "adjoint_backward")
        return {"dl_dms": gms, "dl_dh_ext": ge, "dl_dh_ac": ga, "dl_dm0": g0}

    # -- transfers --
    def copy_field(self, observable: int, dtype=np.float64, out: Optional[np.ndarray] = None) -> np.ndarray:
        """AoS copy of a field.  `out`: a caller-owned contiguous array of 3N
        elements of `dtype` to fill (pinned memory makes the device-to-host copy
        run at full speed); otherwise a new array."""
        if out is None:
            out = np.empty(3 * self.n, dtype=dtype)
        elif out.dtype != dtype or out.size != 3 * self.n or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"out must be a contiguous {np.dtype(dtype).name} array of {3 * self.n} elements")
        if dtype == np.float64:
            rc = self._lib.fullmag_fdm_backend_copy_field_f64(self._h, observable, out.ctypes.data_as(_dp), out.size)
        else:
            rc = self._lib.fullmag_fdm_backend_copy_field_f32(
                self._h, observable, out.ctypes.data_as(C.POINTER(C.c_float)), out.size)
        self._check(rc, "copy_field")
        return out

    def copy_m(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        return self.copy_field(OBS_M, out=out)

    def copy_preview(self, observable: int, preview: Tuple[int, int, int], z_origin: int = 0,
                     z_stride: int = 1, dtype=np.float64) -> np.ndarray:
        pnx, pny, pnz = preview
        out = np.zeros(3 * pnx * pny * pnz, dtype=dtype)
        fn = (self._lib.fullmag_fdm_backend_copy_field_preview_f64 if dtype == np.float64
              else self._lib.fullmag_fdm_backend_copy_field_preview_f32)
        ptr = out.ctypes.data_as(_dp if dtype == np.float64 else C.POINTER(C.c_float))
        self._check(fn(self._h, observable, pnx, pny, pnz, z_origin, z_stride, ptr, out.size), "preview")
        return out

    def snapshot(self, observable: int) -> np.ndarray:
        snap = self._lib.fullmag_fdm_backend_begin_field_snapshot(self._h, observable)
        if not snap:
            err = self._lib.fullmag_fdm_backend_last_error(self._h)
            raise RunError(f"snapshot failed: {err.decode() if err else 'unknown'}")
        try:
            data = C.c_void_p()
            nbytes = C.c_uint64()
            desc = SnapshotDesc()
            rc = self._lib.fullmag_fdm_field_snapshot_wait(snap, C.byref(data), C.byref(nbytes), C.byref(desc))
            if rc != OK:
                raise RunError(f"snapshot wait failed ({rc})")
            dt = np.float32 if desc.scalar_type == SNAP_F32 else np.float64
            buf = (C.c_char * nbytes.value).from_address(data.value)
            return np.frombuffer(bytes(buf), dtype=dt).reshape(3, desc.cell_count).copy()
        finally:
            self._lib.fullmag_fdm_field_snapshot_destroy(snap)

    def upload_m(self, m_aos: np.ndarray) -> None:
        m = np.ascontiguousarray(m_aos).reshape(-1)
        if m.dtype == np.float32:
            rc = self._lib.fullmag_fdm_backend_upload_magnetization_f32(
                self._h, m.ctypes.data_as(C.POINTER(C.c_float)), m.size)
        else:
            m = m.astype(np.float64, copy=False)
            rc = self._lib.fullmag_fdm_backend_upload_magnetization_f64(self._h, m.ctypes.data_as(_dp), m.size)
        self._check(rc, "upload_magnetization")

    def refresh_observables(self) -> None:
        self._check(self._lib.fullmag_fdm_backend_refresh_observables(self._h), "refresh_observables")

    def device_info(self) -> dict:
        info = DeviceInfo()
        self._check(self._lib.fullmag_fdm_backend_get_device_info(self._h, C.byref(info)), "device_info")
        return {"name": info.name.decode(), "cc": (info.compute_capability_major, info.compute_capability_minor),
                "driver_version": info.driver_version, "runtime_version": info.runtime_version}

    # -- extension: profiling / memory --
    def set_profiling(self, on: bool) -> None:
        self._lib.fullmag_fdm_backend_set_profiling(self._h, int(on))

    def profile(self) -> dict:
        out = {}
        for i in range(self._lib.fullmag_fdm_backend_profile_count(self._h)):
            name = C.c_char_p()
            ms = C.c_double()
            cnt = C.c_uint64()
            self._lib.fullmag_fdm_backend_profile_entry(self._h, i, C.byref(name), C.byref(ms), C.byref(cnt))
            out[name.value.decode()] = (ms.value, cnt.value)
        return out

    def profile_reset(self) -> None:
        self._lib.fullmag_fdm_backend_profile_reset(self._h)

    def stream(self) -> int:
        p = C.c_void_p()
        self._check(self._lib.fullmag_fdm_backend_get_stream(self._h, C.byref(p)), "get_stream")
        return int(p.value or 0)

    def memory_info(self) -> Tuple[int, Tuple[int, int, int]]:
        b = C.c_uint64()
        dims = (C.c_uint32 * 3)()
        self._lib.fullmag_fdm_backend_memory_info(self._h, C.byref(b), dims)
        return b.value, tuple(dims)


class NativeFdmBatch:
    """Many independent uniform-material problems stepped together with Heun
    (fullmag_fdm_batch_*).  `problems` is a list of dicts with keys cells,
    cell_size, ms, aex, alpha, gamma, h_ext (A/m) and m0 (AoS 3N)."""

    def __init__(self, problems, precision: int = PRECISION_SINGLE):
        self._lib = load_library()
        arr = (BatchProblem * len(problems))()
        self._keep = []
        self.sizes = []
        for i, p in enumerate(problems):
            nx, ny, nz = (int(v) for v in p["cells"])
            b = arr[i]
            b.nx, b.ny, b.nz = nx, ny, nz
            b.dx, b.dy, b.dz = (float(v) for v in p["cell_size"])
            b.saturation_magnetisation = float(p["ms"])
            b.exchange_stiffness = float(p["aex"])
            b.damping = float(p["alpha"])
            b.gyromagnetic_ratio = float(p.get("gamma", 2.211e5))
            for c, v in enumerate(p.get("h_ext", (0.0, 0.0, 0.0))):
                b.external_field_am[c] = float(v)
            m0 = np.ascontiguousarray(p["m0"], dtype=np.float64).reshape(-1)
            assert m0.size == 3 * nx * ny * nz
            self._keep.append(m0)
            b.initial_magnetization_xyz = m0.ctypes.data_as(_dp)
            self.sizes.append(nx * ny * nz)
        self._h = self._lib.fullmag_fdm_batch_create(arr, len(problems), precision)
        if not self._h:
            raise RunError("fullmag_fdm_batch_create returned NULL")
        err = self._lib.fullmag_fdm_batch_last_error(self._h)
        if err:
            self.close()
            raise RunError(err.decode())

    def _check(self, rc: int, what: str):
        if rc != OK:
            err = self._lib.fullmag_fdm_batch_last_error(self._h)
            raise RunError(f"{what}: {err.decode() if err else rc}")

    def step_n(self, dt: float, n: int) -> None:
        self._check(self._lib.fullmag_fdm_batch_step_n(self._h, dt, n), "batch_step_n")

    def copy_m(self, index: int) -> np.ndarray:
        out = np.zeros(3 * self.sizes[index])
        self._check(self._lib.fullmag_fdm_batch_copy_m(self._h, index, out.ctypes.data_as(_dp), out.size),
                    "batch_copy_m")
        return out

    def stream(self) -> int:
        p = C.c_void_p()
        self._check(self._lib.fullmag_fdm_batch_get_stream(self._h, C.byref(p)), "batch_get_stream")
        return int(p.value or 0)

    def profile_step(self, dt: float) -> list:
        """One step, launches timed by kind (ms): x fwd, y fwd, z, y inv, x inv, stage, predictor."""
        ms = (C.c_float * 7)()
        self._check(self._lib.fullmag_fdm_batch_profile_step(self._h, dt, ms, 7), "batch_profile_step")
        return [float(v) for v in ms]

    def tuning(self):
        """The autotuner's picks: 7 grid sizes (x fwd, y fwd, z, y inv, x inv,
        stage, predictor), then the x and y passes' threads per block."""
        g = (C.c_int32 * 9)()
        self._check(self._lib.fullmag_fdm_batch_tuning(self._h, g, 9), "batch_tuning")
        return list(g)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.fullmag_fdm_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()
