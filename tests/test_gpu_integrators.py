"""GPU parity of the RK4, RK23 (Bogacki-Shampine) and ABM3 integrators
(crates/fullmag-engine/src/lib.rs:1253-1407, 1573-1648) through the C ABI,
against the FP64 oracle.

Tolerances: FP64 max|dm| <= 1e-10 and energies relative 1e-9 (as for Heun and
DP45); RK23's accepted dt and suggested dt relative 1e-9 / 1e-6; FP32-mixed
vs the FP64 oracle max|dm| <= 1e-5 inside the predictability horizon.
"""
import numpy as np
import pytest

from fullmag_b200 import native_fdm as nf

from gpu_helpers import MU0, c1_kwargs, make_pair, max_abs, rel

pytestmark = pytest.mark.gpu


def _energy_close(st, r, tol):
    assert rel(st["exchange_energy_joules"], r["e_ex_pair"]) <= tol
    assert rel(st["demag_energy_joules"], r["e_demag"]) <= tol
    assert rel(st["max_effective_field_amplitude"], r["max_h_eff"]) <= tol
    assert rel(st["max_rhs_amplitude"], r["max_rhs"]) <= tol


@pytest.mark.parametrize("integrator", [nf.RK4, nf.ABM3])
def test_fixed_step_fp64_c1_matches_oracle(integrator):
    be, sim, _ = make_pair(**c1_kwargs(), integrator=integrator)
    for i in range(60):
        st = be.step(1e-13)
        r = sim.step(1e-13)
    assert max_abs(be.copy_m(), sim.m) <= 1e-10
    assert st["step"] == 60 and abs(st["time_seconds"] - 6e-12) < 1e-24
    _energy_close(st, r, 1e-9)


@pytest.mark.parametrize("integrator", [nf.RK4, nf.ABM3, nf.RK23])
def test_fp64_3d_smooth_matches_oracle(integrator):
    nx, ny, nz = 24, 12, 4
    x = (np.arange(nx) + 0.5) / nx
    m0 = np.zeros((nz, ny, nx, 3))
    m0[..., 0] = np.cos(0.8 * np.pi * x)
    m0[..., 1] = np.sin(0.8 * np.pi * x)
    m0[..., 2] = 0.2
    m0 /= np.linalg.norm(m0, axis=-1, keepdims=True)
    adaptive = (1e-6, 1e-18, 1e-12, 0.8) if integrator == nf.RK23 else None
    be, sim, _ = make_pair((nx, ny, nz), (2e-9, 2.5e-9, 3e-9), alpha=0.2, h_ext=(2e4, -1e4, 5e3),
                           m0=m0.reshape(-1), integrator=integrator, adaptive=adaptive,
                           symmetric_kernel=True)
    dt = 5e-14
    for _ in range(30):
        st = be.step(dt)
        r = sim.step(dt)
        if integrator == nf.RK23:
            assert rel(st["dt_seconds"], r["dt_used"]) <= 1e-9
            assert rel(st["suggested_next_dt"], r["suggested_next_dt"]) <= 1e-6
            dt = st["suggested_next_dt"]
    assert max_abs(be.copy_m(), sim.m) <= 1e-10
    assert abs(st["time_seconds"] - sim.time) <= 1e-9 * sim.time
    _energy_close(st, r, 1e-9)


def test_rk23_masked_adaptive_matches_oracle():
    """A masked disk, large initial dt: rejected attempts, then the controller's
    dt sequence, like the DP45 test."""
    nx, ny, nz = 32, 32, 2
    xs = (np.arange(nx) + 0.5) * 2e-9 - nx * 1e-9
    xx, yy = np.meshgrid(xs, xs)
    disk = ((xx ** 2 + yy ** 2) <= (30e-9) ** 2) & ((xx ** 2 + yy ** 2) >= (8e-9) ** 2)
    mask = np.repeat(disk[None], nz, axis=0).astype(np.uint8).reshape(-1)
    adaptive = (1e-5, 1e-18, 1e-10, 0.8)
    be, sim, _ = make_pair((nx, ny, nz), (2e-9, 2e-9, 2e-9), alpha=0.1, h_ext=(0, 30e-3 / MU0, 0),
                           mask=mask, integrator=nf.RK23, adaptive=adaptive, seed=44)
    dt = 1e-12
    for _ in range(15):
        st = be.step(dt)
        r = sim.step(dt)
        assert rel(st["dt_seconds"], r["dt_used"]) <= 1e-9
        assert rel(st["suggested_next_dt"], r["suggested_next_dt"]) <= 1e-6
        dt = st["suggested_next_dt"]
    assert max_abs(be.copy_m(), sim.m) <= 1e-10
    _energy_close(st, r, 1e-9)


def test_abm3_dt_change_restarts_like_oracle():
    be, sim, _ = make_pair(**c1_kwargs(), integrator=nf.ABM3)
    for dt in [1e-13] * 6 + [1.5e-13] * 5 + [1.52e-13] * 4:
        st = be.step(dt)
        r = sim.step(dt)
    assert max_abs(be.copy_m(), sim.m) <= 1e-10
    _energy_close(st, r, 1e-9)


@pytest.mark.parametrize("integrator", [nf.RK4, nf.ABM3, nf.RK23])
def test_fp32_mixed_matches_fp64_oracle(integrator):
    adaptive = (1e-5, 1e-18, 1e-12, 0.8) if integrator == nf.RK23 else None
    be, sim, _ = make_pair(**c1_kwargs(), integrator=integrator, precision=nf.PRECISION_SINGLE,
                           adaptive=adaptive)
    dt = 1e-13
    for _ in range(20):
        st = be.step(dt)
        sim.step(dt)
        if integrator == nf.RK23:
            dt = st["suggested_next_dt"]
    assert max_abs(be.copy_m(), sim.m) <= 1e-5


@pytest.mark.parametrize("integrator", [nf.RK4, nf.ABM3, nf.RK23])
def test_step_n_equals_repeated_steps(integrator):
    adaptive = (1e-6, 1e-18, 1e-12, 0.8) if integrator == nf.RK23 else None
    kw = dict(cells=(32, 16, 2), cell_size=(2e-9, 2e-9, 2e-9), alpha=0.1, h_ext=(1e4, 2e4, 0),
              integrator=integrator, adaptive=adaptive)
    a, _, _ = make_pair(**kw)
    b, _, _ = make_pair(**kw)
    dt = 3e-14
    for _ in range(12):
        sa = a.step(dt)
        if integrator == nf.RK23:
            dt = sa["suggested_next_dt"]
    sb = b.step_n(3e-14, 12)
    assert np.array_equal(a.copy_m(), b.copy_m())
    for k in ("exchange_energy_joules", "demag_energy_joules", "max_rhs_amplitude", "step", "time_seconds"):
        assert sa[k] == sb[k]
