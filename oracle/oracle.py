"""ctypes binding of the FP64 CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference's CPU engine (crates/fullmag-engine) and
Newell tensor (crates/fullmag-fdm-demag/src/newell.rs) in C++; see oracle.h.
Only tests, the smoke check and the CPU-baseline leg of bench.py import this
module.  The product library never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

HEUN = 1
DP45 = 2
ABM3 = 3
RK4 = 4
RK23 = 5


class OracleDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("ms", C.c_double), ("aex", C.c_double), ("alpha", C.c_double), ("gamma", C.c_double),
        ("integrator", C.c_int), ("precession_enabled", C.c_int),
        ("enable_exchange", C.c_int), ("enable_demag", C.c_int),
        ("has_external_field", C.c_int), ("h_ext", C.c_double * 3),
        ("active_mask", C.POINTER(C.c_uint8)), ("region_mask", C.POINTER(C.c_uint32)),
        ("exchange_lut", C.POINTER(C.c_double)), ("ms_map", C.POINTER(C.c_double)),
        ("max_error", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double),
        ("headroom", C.c_double),
        ("h_ac", C.c_double * 3), ("ac_freq", C.c_double),
        ("thin_film_2d", C.c_int), ("symmetric_kernel", C.c_int),
        ("boundary_tier", C.c_int), ("phi_floor", C.c_double), ("delta_min", C.c_double),
        ("volume_fraction", C.POINTER(C.c_double)),
        ("face_link", C.POINTER(C.c_double) * 6), ("delta", C.POINTER(C.c_double) * 6),
        ("corr_target", C.POINTER(C.c_int32)), ("corr_source", C.POINTER(C.c_int32)),
        ("corr_tensor", C.POINTER(C.c_double)),
        ("corr_targets", C.c_uint32), ("corr_stencil", C.c_uint32),
    ]


class OracleReport(C.Structure):
    _fields_ = [
        ("time_seconds", C.c_double), ("dt_used", C.c_double),
        ("e_ex_field", C.c_double), ("e_ex_pair", C.c_double),
        ("e_demag", C.c_double), ("e_ext", C.c_double), ("e_total", C.c_double),
        ("max_h_eff", C.c_double), ("max_h_demag", C.c_double), ("max_rhs", C.c_double),
        ("suggested_next_dt", C.c_double), ("rejected_attempts", C.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def build() -> str:
    """Compile the oracle with its Makefile (g++ -fopenmp) if needed."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.POINTER(OracleDesc), dp]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_step.argtypes = [C.c_void_p, C.c_double, C.POINTER(OracleReport)]
        L.oracle_step.restype = C.c_int
        L.oracle_get_m.argtypes = [C.c_void_p, dp]
        L.oracle_set_m.argtypes = [C.c_void_p, dp]
        L.oracle_time.argtypes = [C.c_void_p]
        L.oracle_time.restype = C.c_double
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_observe.argtypes = [C.c_void_p, dp, dp, dp, dp, dp, C.POINTER(OracleReport)]
        L.oracle_newell_kernels.argtypes = [C.c_uint32] * 3 + [C.c_double] * 3 + [dp]
        L.oracle_newell_spectra.argtypes = [C.c_uint32] * 3 + [C.c_double] * 3 + [C.c_int] + [dp] * 6
        L.oracle_newell_f.restype = C.c_double
        L.oracle_newell_f.argtypes = [C.c_double] * 3
        L.oracle_newell_g.restype = C.c_double
        L.oracle_newell_g.argtypes = [C.c_double] * 3
        L.oracle_fft.argtypes = [dp, C.c_uint64, C.c_int]
        L.oracle_random_unit_vectors.argtypes = [C.c_uint64, C.c_uint64, dp]
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def fft(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().oracle_fft(a.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)), a.size, int(inverse))
    return a


def newell_f(x, y, z) -> float:
    return lib().oracle_newell_f(x, y, z)


def newell_g(x, y, z) -> float:
    return lib().oracle_newell_g(x, y, z)


def newell_kernels(nx, ny, nz, dx, dy, dz) -> np.ndarray:
    """Real-space tensor, shape (6, 2nz, 2ny, 2nx): xx, yy, zz, xy, xz, yz."""
    p = 8 * nx * ny * nz
    out = np.zeros(6 * p)
    lib().oracle_newell_kernels(nx, ny, nz, dx, dy, dz, _dptr(out))
    return out.reshape(6, 2 * nz, 2 * ny, 2 * nx)


def newell_spectra(nx, ny, nz, dx, dy, dz, thin_film_2d=False):
    """Interleaved complex spectra [2P] per component, as the reference host passes them."""
    pz = 1 if thin_film_2d else 2 * nz
    p = 2 * nx * 2 * ny * pz
    outs = [np.zeros(2 * p) for _ in range(6)]
    lib().oracle_newell_spectra(nx, ny, nz, dx, dy, dz, int(thin_film_2d), *[_dptr(o) for o in outs])
    return outs


def random_unit_vectors(seed: int, count: int) -> np.ndarray:
    out = np.zeros(3 * count)
    lib().oracle_random_unit_vectors(seed, count, _dptr(out))
    return out


@dataclass
class Problem:
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    ms: float = 8.0e5
    aex: float = 1.3e-11
    alpha: float = 0.02
    gamma: float = 2.211e5
    integrator: int = HEUN
    precession: bool = True
    exchange: bool = True
    demag: bool = True
    h_ext: Optional[Sequence[float]] = None
    active_mask: Optional[np.ndarray] = None
    region_mask: Optional[np.ndarray] = None
    exchange_lut: Optional[np.ndarray] = None
    ms_map: Optional[np.ndarray] = None
    max_error: float = 0.0
    dt_min: float = 0.0
    dt_max: float = 0.0
    headroom: float = 0.0
    h_ac: Optional[Sequence[float]] = None
    ac_freq: float = 0.0
    thin_film_2d: bool = False
    symmetric_kernel: bool = False
    # boundary tiers: 0 none, 1 T0, 2 T1; arrays [N], directions xp, xm, yp, ym, zp, zm
    boundary_tier: int = 0
    phi_floor: float = 0.0
    delta_min: float = 0.0
    volume_fraction: Optional[np.ndarray] = None
    face_link: Optional[Sequence[np.ndarray]] = None
    delta: Optional[Sequence[np.ndarray]] = None
    corr_target: Optional[np.ndarray] = None
    corr_source: Optional[np.ndarray] = None   # [T, S]
    corr_tensor: Optional[np.ndarray] = None   # [T, S, 6] xx, xy, xz, yy, yz, zz
    _keep: list = field(default_factory=list, repr=False)

    def desc(self) -> OracleDesc:
        d = OracleDesc()
        d.nx, d.ny, d.nz = self.nx, self.ny, self.nz
        d.dx, d.dy, d.dz = self.dx, self.dy, self.dz
        d.ms, d.aex, d.alpha, d.gamma = self.ms, self.aex, self.alpha, self.gamma
        d.integrator = self.integrator
        d.precession_enabled = int(self.precession)
        d.enable_exchange = int(self.exchange)
        d.enable_demag = int(self.demag)
        d.has_external_field = int(self.h_ext is not None)
        for i, v in enumerate(self.h_ext or (0.0, 0.0, 0.0)):
            d.h_ext[i] = v
        for i, v in enumerate(self.h_ac or (0.0, 0.0, 0.0)):
            d.h_ac[i] = v
        d.ac_freq = self.ac_freq
        self._keep = []
        if self.active_mask is not None:
            a = np.ascontiguousarray(self.active_mask, dtype=np.uint8)
            self._keep.append(a)
            d.active_mask = a.ctypes.data_as(C.POINTER(C.c_uint8))
        if self.region_mask is not None:
            a = np.ascontiguousarray(self.region_mask, dtype=np.uint32)
            self._keep.append(a)
            d.region_mask = a.ctypes.data_as(C.POINTER(C.c_uint32))
        if self.exchange_lut is not None:
            a = np.ascontiguousarray(self.exchange_lut, dtype=np.float64)
            self._keep.append(a)
            d.exchange_lut = _dptr(a)
        if self.ms_map is not None:
            a = np.ascontiguousarray(self.ms_map, dtype=np.float64)
            self._keep.append(a)
            d.ms_map = _dptr(a)
        d.max_error, d.dt_min, d.dt_max, d.headroom = (
            self.max_error, self.dt_min, self.dt_max, self.headroom)
        d.thin_film_2d = int(self.thin_film_2d)
        d.symmetric_kernel = int(self.symmetric_kernel)
        d.boundary_tier = int(self.boundary_tier)
        d.phi_floor, d.delta_min = self.phi_floor, self.delta_min

        def keep_d(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            self._keep.append(a)
            return _dptr(a)

        def keep_i(a):
            a = np.ascontiguousarray(a, dtype=np.int32)
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_int32))

        if self.volume_fraction is not None:
            d.volume_fraction = keep_d(self.volume_fraction)
        for q in range(6):
            if self.face_link is not None:
                d.face_link[q] = keep_d(self.face_link[q])
            if self.delta is not None:
                d.delta[q] = keep_d(self.delta[q])
        if self.corr_target is not None:
            t = np.asarray(self.corr_target)
            src = np.asarray(self.corr_source)
            d.corr_target = keep_i(t)
            d.corr_source = keep_i(src.reshape(-1))
            d.corr_tensor = keep_d(np.asarray(self.corr_tensor).reshape(-1))
            d.corr_targets = t.size
            d.corr_stencil = src.size // max(t.size, 1)
        return d


class Simulation:
    """One oracle problem + state (ExchangeLlgProblem + ExchangeLlgState + workspace)."""

    def __init__(self, problem: Problem, m0_aos: np.ndarray):
        self.problem = problem
        self.n = problem.nx * problem.ny * problem.nz
        m0 = np.ascontiguousarray(m0_aos, dtype=np.float64).reshape(-1)
        assert m0.size == 3 * self.n
        self._desc = problem.desc()
        self._h = lib().oracle_create(C.byref(self._desc), _dptr(m0))
        if not self._h:
            raise ValueError("oracle_create failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().oracle_destroy(h)
            self._h = None

    def step(self, dt: float) -> dict:
        r = OracleReport()
        rc = lib().oracle_step(self._h, dt, C.byref(r))
        if rc != 0:
            raise ValueError("oracle_step failed")
        return r.as_dict()

    @property
    def m(self) -> np.ndarray:
        out = np.zeros(3 * self.n)
        lib().oracle_get_m(self._h, _dptr(out))
        return out

    def set_m(self, m_aos: np.ndarray) -> None:
        a = np.ascontiguousarray(m_aos, dtype=np.float64).reshape(-1)
        lib().oracle_set_m(self._h, _dptr(a))

    @property
    def time(self) -> float:
        return lib().oracle_time(self._h)

    def observe(self) -> dict:
        bufs = {k: np.zeros(3 * self.n) for k in ("h_ex", "h_demag", "h_ext", "h_eff", "rhs")}
        r = OracleReport()
        lib().oracle_observe(self._h, *[_dptr(bufs[k]) for k in ("h_ex", "h_demag", "h_ext", "h_eff", "rhs")],
                             C.byref(r))
        out = r.as_dict()
        out.update(bufs)
        return out
