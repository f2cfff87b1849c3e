"""GPU parity against the FP64 oracle at the sizes the benchmark is quoted on.

C2 exactly: 512 x 512 x 8 film of 2 nm cells, Ms 8e5 A/m, A 1.3e-11 J/m,
alpha 0.5, B = (10, 0, 0) mT, m0 from the planner generator with seed 43, the
library's own Newell spectra.  That is the grid of the throughput benchmark,
with its 1024-point x and y lines and the fused kx-plane pass (FP32) or the
split y passes with the direct z sum (FP64).

Reduced C3: the C3 geometry (disk of radius 1 um with a centred hole of
radius 150 nm, Ms = 0 outside, 2 nm cells, alpha 0.1, B = (0, 30, 0) mT,
seed 44) cut to a band of the grid that keeps C3's kernel selection:
1024 x 64 x 16 keeps the 2048-point x lines, 32 x 1024 x 16 the 2048-point y
lines, and both have nz = 16 (the z FFT pass, not the direct sum) and the
masked stage kernels.  DP45 at max_error 1e-5 feeding back the suggested dt.

Tolerances:
  - FP64 fields 1e-13 of each field's max |H| (the oracle convolves with the
    exactly even/odd spectra the library stores); FP64 trajectories 1e-12
    (C2, 2 Heun steps) and 1e-10 (C3 band, DP45), the DP45 dt sequence 1e-9;
  - FP32-mixed fields 2e-6 of max |H|, C2 trajectories 1e-6 after 2 steps;
  - FP32-mixed DP45 on the C3 band: with dt held fixed (dt_min = dt_max) the
    state is compared at 1e-5 (the reference's tier-B bound,
    native/backends/fdm/tests/tier_b_compare.cu:113-114).  Adaptively, the
    error norm of random-m0 stages cancels ~1e4-fold, so FP32 rounding moves
    the norm by ~1e-3 relative and the dt by ~1e-4; the accepted dt sequence is
    compared with FP64's at 1e-2 relative and the states are reported.
"""
import os

import numpy as np
import pytest

from fullmag_b200 import native_fdm as nf
from oracle import oracle as O

from gpu_helpers import MU0, max_abs

pytestmark = pytest.mark.gpu


def _threads():
    O.set_threads(os.cpu_count() or 1)


def _field_errors(be, obs):
    out = {}
    for o, key in ((nf.OBS_H_EX, "h_ex"), (nf.OBS_H_DEMAG, "h_demag"), (nf.OBS_H_EFF, "h_eff")):
        ref = obs[key]
        out[key] = max_abs(be.copy_field(o), ref) / max(np.abs(ref).max(), 1e-300)
    return out


def _disk_band(nx, ny, nz, d, r_out=1e-6, r_in=150e-9):
    """The C3 disk-with-hole mask (cell-centre test) on an nx x ny band centred
    on the disk."""
    x = (np.arange(nx) + 0.5) * d - nx * d / 2
    y = (np.arange(ny) + 0.5) * d - ny * d / 2
    X, Y = np.meshgrid(x, y)
    r2 = X ** 2 + Y ** 2
    m2 = (r2 <= r_out ** 2) & (r2 > r_in ** 2)
    return np.repeat(m2[None], nz, axis=0).astype(np.uint8).reshape(-1)


def test_c2_fields_and_heun_steps_match_oracle():
    _threads()
    nx, ny, nz, d = 512, 512, 8, 2e-9
    n = nx * ny * nz
    h = (10e-3 / MU0, 0.0, 0.0)
    m0 = O.random_unit_vectors(43, n)
    prob = O.Problem(nx, ny, nz, d, d, d, ms=8e5, aex=1.3e-11, alpha=0.5, gamma=2.211e5, h_ext=h,
                     symmetric_kernel=True)
    sim = O.Simulation(prob, m0)
    obs = sim.observe()
    ref_m = []
    for _ in range(2):
        sim.step(5e-14)
        ref_m.append(sim.m.copy())
    for prec, ftol, mtol in ((nf.PRECISION_DOUBLE, 1e-13, 1e-12), (nf.PRECISION_SINGLE, 2e-6, 1e-6)):
        plan = nf.FdmPlan(cells=(nx, ny, nz), cell_size=(d, d, d), initial_magnetization=m0,
                          saturation_magnetisation=8e5, exchange_stiffness=1.3e-11, damping=0.5,
                          gyromagnetic_ratio=2.211e5, precision=prec, external_field=h,
                          demag_source=nf.DEMAG_NEWELL)
        be = nf.NativeFdmBackend(plan)
        err = _field_errors(be, obs)
        dms = []
        for k in range(2):
            be.step(5e-14)
            dms.append(max_abs(be.copy_m(), ref_m[k]))
        be.close()
        print(f"C2 precision {prec}: fields", {k: f"{v:.2e}" for k, v in err.items()},
              "max|dm| after 1, 2 steps:", [f"{v:.2e}" for v in dms])
        for k, v in err.items():
            assert v <= ftol, (prec, k, v)
        for v in dms:
            assert v <= mtol, (prec, dms)


C3_BANDS = [(1024, 64, 16), (32, 1024, 16)]


def _c3_plan(cells, m0, mask, prec, adaptive):
    d = 2e-9
    return nf.FdmPlan(cells=cells, cell_size=(d, d, d), initial_magnetization=m0,
                      saturation_magnetisation=8e5, exchange_stiffness=1.3e-11, damping=0.1,
                      gyromagnetic_ratio=2.211e5, precision=prec, integrator=nf.DP45,
                      external_field=(0.0, 30e-3 / MU0, 0.0), active_mask=mask, adaptive=adaptive,
                      demag_source=nf.DEMAG_NEWELL)


def _c3_oracle(cells, m0, mask, adaptive):
    d = 2e-9
    prob = O.Problem(*cells, d, d, d, ms=8e5, aex=1.3e-11, alpha=0.1, gamma=2.211e5,
                     integrator=O.DP45, h_ext=(0.0, 30e-3 / MU0, 0.0), active_mask=mask,
                     symmetric_kernel=True)
    prob.max_error, prob.dt_min, prob.dt_max, prob.headroom = adaptive
    return O.Simulation(prob, m0)


@pytest.mark.parametrize("cells", C3_BANDS)
def test_c3_band_masked_dp45_fp64_matches_oracle(cells):
    _threads()
    nx, ny, nz = cells
    mask = _disk_band(nx, ny, nz, 2e-9)
    m0 = O.random_unit_vectors(44, nx * ny * nz)
    adaptive = (1e-5, 1e-18, 1e-10, 0.8)
    sim = _c3_oracle(cells, m0, mask, adaptive)
    obs = sim.observe()
    be = nf.NativeFdmBackend(_c3_plan(cells, m0, mask, nf.PRECISION_DOUBLE, adaptive))
    err = _field_errors(be, obs)
    print(cells, "FP64 fields:", {k: f"{v:.2e}" for k, v in err.items()})
    for k, v in err.items():
        assert v <= 1e-13, (k, v)
    dt = 1e-13
    for s in range(3):
        st = be.step(dt)
        r = sim.step(dt)
        dm = max_abs(be.copy_m(), sim.m)
        print(f"{cells} FP64 DP45 step {s + 1}: dt {st['dt_seconds']:.6e} (oracle {r['dt_used']:.6e}), "
              f"max|dm| {dm:.2e}")
        assert abs(st["dt_seconds"] - r["dt_used"]) <= 1e-9 * r["dt_used"]
        assert abs(st["suggested_next_dt"] - r["suggested_next_dt"]) <= 1e-6 * r["suggested_next_dt"]
        assert dm <= 1e-10, (s, dm)
        dt = st["suggested_next_dt"]
    m = be.copy_m().reshape(-1, 3)
    assert np.all(m[mask == 0] == 0.0)
    be.close()


@pytest.mark.parametrize("cells", C3_BANDS)
def test_c3_band_masked_dp45_fp32_mixed(cells):
    _threads()
    nx, ny, nz = cells
    mask = _disk_band(nx, ny, nz, 2e-9)
    m0 = O.random_unit_vectors(44, nx * ny * nz)
    # dt held fixed: the FP32-mixed stages against the FP64 oracle on the same dt
    fixed = (1e-5, 2e-14, 2e-14, 0.8)
    sim = _c3_oracle(cells, m0, mask, fixed)
    obs = sim.observe()
    be = nf.NativeFdmBackend(_c3_plan(cells, m0, mask, nf.PRECISION_SINGLE, fixed))
    err = _field_errors(be, obs)
    print(cells, "FP32-mixed fields:", {k: f"{v:.2e}" for k, v in err.items()})
    for k, v in err.items():
        assert v <= 2e-6, (k, v)
    for s in range(3):
        be.step(2e-14)
        sim.step(2e-14)
        dm = max_abs(be.copy_m(), sim.m)
        print(f"{cells} FP32-mixed DP45 at fixed dt 2e-14, step {s + 1}: max|dm| {dm:.2e}")
        assert dm <= 1e-5, (s, dm)
    be.close()
    # adaptive: FP32-mixed and FP64 on the same schedule of suggested dt
    adaptive = (1e-5, 1e-18, 1e-10, 0.8)
    b32 = nf.NativeFdmBackend(_c3_plan(cells, m0, mask, nf.PRECISION_SINGLE, adaptive))
    b64 = nf.NativeFdmBackend(_c3_plan(cells, m0, mask, nf.PRECISION_DOUBLE, adaptive))
    d32 = d64 = 1e-13
    for s in range(3):
        s32, s64 = b32.step(d32), b64.step(d64)
        dm = max_abs(b32.copy_m(), b64.copy_m())
        print(f"{cells} adaptive step {s + 1}: dt FP32 {s32['dt_seconds']:.6e} FP64 {s64['dt_seconds']:.6e}, "
              f"max|m32 - m64| {dm:.2e}")
        assert abs(s32["dt_seconds"] - s64["dt_seconds"]) <= 1e-2 * s64["dt_seconds"]
        d32, d64 = s32["suggested_next_dt"], s64["suggested_next_dt"]
    b32.close()
    b64.close()
