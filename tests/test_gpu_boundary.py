"""GPU parity of the boundary tiers through the C ABI against the FP64 oracle:
T0 (face-link exchange, native/backends/fdm/src/exchange_t0_fp64.cu), T1 (ECB
stencil, exchange_t1_fp64.cu), the phi-weighted demag packing
(demag_fp64.cu:79-85) and the sparse demag correction (demag_boundary_fp64.cu).

Tolerances as in test_gpu_parity.py: FP64 fields 1e-13 of each field's max
against the symmetric-kernel oracle, trajectories 1e-10, energies 1e-9;
FP32-mixed fields 2e-6 and trajectories 1e-5.
"""
import numpy as np
import pytest

from fullmag_b200 import native_fdm as nf

from boundary_geometry import disk_geometry
from gpu_helpers import make_pair, max_abs, rel

pytestmark = pytest.mark.gpu

CELLS = (24, 24, 2)
SIZE = (3e-9, 3e-9, 3e-9)


def _geometry(tier, corr=True, faces=True, deltas=True):
    g = disk_geometry(*CELLS, *SIZE, radius=31e-9)
    return g, dict(tier=tier, vf=g["vf"], faces=g["faces"] if faces else None,
                   deltas=g["deltas"] if deltas else None, corr=g["corr"] if corr else None)


def _field_errors(be, obs):
    out = {}
    for o, key in ((nf.OBS_H_EX, "h_ex"), (nf.OBS_H_DEMAG, "h_demag"), (nf.OBS_H_EFF, "h_eff")):
        ref = obs[key]
        out[key] = max_abs(be.copy_field(o), ref) / max(np.abs(ref).max(), 1e-300)
    return out


@pytest.mark.parametrize("tier", [nf.BOUNDARY_VOLUME, nf.BOUNDARY_FULL])
@pytest.mark.parametrize("fft", ["register", "stockham"])
def test_tier_fields_and_heun_trajectory_fp64(monkeypatch, tier, fft):
    if fft == "stockham":
        monkeypatch.setenv("FULLMAG_FDM_FFT", "stockham")
    else:
        monkeypatch.delenv("FULLMAG_FDM_FFT", raising=False)
    g, bnd = _geometry(tier)
    be, sim, _ = make_pair(CELLS, SIZE, alpha=0.1, h_ext=(2e4, 1e4, 0), mask=g["mask"], seed=21,
                           symmetric_kernel=True, boundary=bnd)
    err = _field_errors(be, sim.observe())
    print(tier, fft, {k: f"{v:.2e}" for k, v in err.items()})
    for k, v in err.items():
        assert v <= 1e-13, (k, v)
    for _ in range(30):
        st = be.step(5e-14)
        r = sim.step(5e-14)
    assert max_abs(be.copy_m(), sim.m) <= 1e-10
    assert rel(st["demag_energy_joules"], r["e_demag"]) <= 1e-9
    assert rel(st["exchange_energy_joules"], r["e_ex_pair"]) <= 1e-9


def test_tier_launch_conditions_follow_the_reference():
    """T1 without distances keeps the standard exchange (and the phi-weighted
    demag); T0 without face links likewise (exchange_fp64.cu:159-198)."""
    for tier, kw in ((nf.BOUNDARY_FULL, dict(deltas=False)), (nf.BOUNDARY_VOLUME, dict(faces=False))):
        g, bnd = _geometry(tier, corr=False, **kw)
        be, sim, _ = make_pair(CELLS, SIZE, alpha=0.1, h_ext=(2e4, 1e4, 0), mask=g["mask"], seed=22,
                               symmetric_kernel=True, boundary=bnd)
        for k, v in _field_errors(be, sim.observe()).items():
            assert v <= 1e-13, (tier, k, v)


@pytest.mark.parametrize("tier", [nf.BOUNDARY_VOLUME, nf.BOUNDARY_FULL])
def test_tier_fp32_mixed_vs_fp64_oracle(tier):
    g, bnd = _geometry(tier)
    be, sim, _ = make_pair(CELLS, SIZE, alpha=0.1, h_ext=(2e4, 1e4, 0), mask=g["mask"], seed=23,
                           symmetric_kernel=True, boundary=bnd, precision=nf.PRECISION_SINGLE)
    for k, v in _field_errors(be, sim.observe()).items():
        assert v <= 2e-6, (k, v)
    for _ in range(20):
        be.step(5e-14)
        sim.step(5e-14)
    assert max_abs(be.copy_m(), sim.m) <= 1e-5


def test_tier_with_rk4_and_dp45():
    g, bnd = _geometry(nf.BOUNDARY_FULL)
    for integ, adaptive in ((nf.RK4, None), (nf.DP45, (1e-5, 1e-18, 1e-12, 0.8))):
        be, sim, _ = make_pair(CELLS, SIZE, alpha=0.1, h_ext=(2e4, 1e4, 0), mask=g["mask"], seed=24,
                               symmetric_kernel=True, boundary=bnd, integrator=integ, adaptive=adaptive)
        dt = 5e-14
        for _ in range(10):
            st = be.step(dt)
            sim.step(dt)
            if integ == nf.DP45:
                dt = st["suggested_next_dt"]
        assert max_abs(be.copy_m(), sim.m) <= 1e-10, integ
