"""The fused row pass (x inverse + stage + x forward per row slab) against the
split kernels it replaces.

In FP64 the row pass runs the operations of the split x inverse, stage and x
forward kernels in the same order; the compiler may still contract a multiply
and an add into one FMA differently in the two kernels, so states are compared
at 1e-13 after one step and 1e-11 after 40 (statistics to 1e-12 relative: the
diagnostics are summed in another order).  In FP32-mixed the row pass
evaluates the stencil and RHS in FP32 (the split stage kernels in FP64), so it
is compared with the FP64 oracle at the FP32-mixed bound of the other parity
tests (1e-5), and so is its difference to the split FP32-mixed path.  Fields read after fused steps
(H_d is never written by them) must equal the split path's, and reading them
must not change the trajectory.
"""
import os

import numpy as np
import pytest

from fullmag_b200 import native_fdm as nf
from oracle import oracle as O

from gpu_helpers import MU0, make_pair, max_abs

pytestmark = pytest.mark.gpu


def _backend(cells, cell_size, prec, row, m0, alpha=0.5, h=(10e-3 / MU0, 0, 0)):
    old = os.environ.get("FULLMAG_FDM_ROW")
    os.environ["FULLMAG_FDM_ROW"] = "on" if row else "off"
    try:
        plan = nf.FdmPlan(cells=cells, cell_size=cell_size, initial_magnetization=m0,
                          saturation_magnetisation=8e5, exchange_stiffness=1.3e-11, damping=alpha,
                          gyromagnetic_ratio=2.211e5, precision=prec, external_field=h,
                          demag_source=nf.DEMAG_NEWELL)
        return nf.NativeFdmBackend(plan)
    finally:
        if old is None:
            del os.environ["FULLMAG_FDM_ROW"]
        else:
            os.environ["FULLMAG_FDM_ROW"] = old


GRIDS = [((64, 16, 1), (3.125e-9, 3.125e-9, 3e-9)),   # thin film, 2-D y pass
         ((32, 32, 4), (2e-9, 2e-9, 2e-9)),           # direct z sum
         ((64, 8, 8), (2e-9, 2.5e-9, 2e-9)),
         ((128, 64, 2), (2e-9, 2e-9, 3e-9))]


@pytest.mark.parametrize("cells,d", GRIDS)
def test_row_pass_fp64_matches_split(cells, d):
    n = cells[0] * cells[1] * cells[2]
    m0 = nf.random_unit_vectors(7, n)
    fused = _backend(cells, d, nf.PRECISION_DOUBLE, True, m0)
    split = _backend(cells, d, nf.PRECISION_DOUBLE, False, m0)
    fused.step(4e-14)
    split.step(4e-14)
    d1 = max_abs(fused.copy_m(), split.copy_m())
    for k in range(39):
        sf = fused.step(4e-14)
        ss = split.step(4e-14)
    d40 = max_abs(fused.copy_m(), split.copy_m())
    print(f"{cells} FP64 row pass vs split: max|dm| after 1 step {d1:.2e}, after 40 {d40:.2e}")
    assert d1 <= 1e-13 and d40 <= 1e-11, (d1, d40)
    for key in ("exchange_energy_joules", "demag_energy_joules", "external_energy_joules",
                "max_effective_field_amplitude", "max_demag_field_amplitude", "max_rhs_amplitude"):
        assert abs(sf[key] - ss[key]) <= 1e-12 * max(abs(ss[key]), 1e-300), (key, sf[key], ss[key])
    # fields after fused steps (H_d recomputed on request)
    for obs in (nf.OBS_H_DEMAG, nf.OBS_H_EX, nf.OBS_H_EFF):
        f, r = fused.copy_field(obs), split.copy_field(obs)
        assert max_abs(f, r) <= 1e-9 * np.abs(r).max(), obs
    # a field read in between does not change the fused trajectory
    m_before = fused.copy_m()
    ref = _backend(cells, d, nf.PRECISION_DOUBLE, True, m0)
    ref.step_n(4e-14, 40)
    assert np.array_equal(ref.copy_m(), m_before)
    for be in (fused, ref):
        be.step_n(4e-14, 5)
    assert np.array_equal(fused.copy_m(), ref.copy_m())
    ref.close()
    fused.close()
    split.close()


@pytest.mark.parametrize("cells,d", GRIDS)
def test_row_pass_fp32_mixed_vs_oracle_and_split(cells, d):
    nx, ny, nz = cells
    n = nx * ny * nz
    m0 = O.random_unit_vectors(43, n)
    h = (10e-3 / MU0, 0.0, 0.0)
    prob = O.Problem(nx, ny, nz, *d, ms=8e5, aex=1.3e-11, alpha=0.5, gamma=2.211e5, h_ext=h,
                     thin_film_2d=False, symmetric_kernel=True)
    sim = O.Simulation(prob, m0)
    fused = _backend(cells, d, nf.PRECISION_SINGLE, True, m0, h=h)
    split = _backend(cells, d, nf.PRECISION_SINGLE, False, m0, h=h)
    for _ in range(50):
        st = fused.step(5e-14)
        split.step(5e-14)
        r = sim.step(5e-14)
    mf = fused.copy_m()
    d_oracle = max_abs(mf, sim.m)
    d_split = max_abs(mf, split.copy_m())
    print(f"{cells} FP32-mixed row pass after 50 steps: vs oracle {d_oracle:.2e}, vs split {d_split:.2e}")
    assert d_oracle <= 1e-5
    assert d_split <= 1e-5
    assert abs(st["total_energy_joules"] - r["e_total"]) <= 1e-4 * abs(r["e_total"])
    hd = fused.copy_field(nf.OBS_H_DEMAG)
    ref = sim.observe()["h_demag"]
    assert max_abs(hd, ref) <= 2e-6 * np.abs(ref).max()
    fused.close()
    split.close()


def test_row_pass_restarts_after_upload_and_dt_change():
    cells, d = (64, 32, 4), (2e-9, 2e-9, 2e-9)
    n = 64 * 32 * 4
    m0 = nf.random_unit_vectors(3, n)
    m1 = nf.random_unit_vectors(4, n)
    fused = _backend(cells, d, nf.PRECISION_DOUBLE, True, m0)
    split = _backend(cells, d, nf.PRECISION_DOUBLE, False, m0)
    for be in (fused, split):
        be.step_n(3e-14, 5)
        be.upload_m(m1)
        be.step_n(3e-14, 3)
        be.step_n(5e-14, 4)   # dt change: the predictor is rebuilt
        be.refresh_observables()
        be.step_n(5e-14, 2)
    dm = max_abs(fused.copy_m(), split.copy_m())
    print(f"row pass after upload / dt change / refresh vs split: {dm:.2e}")
    assert dm <= 1e-11
    fused.close()
    split.close()
