"""C3 at its full size: the 1024 x 1024 x 16 masked FP32-mixed DP45 run.

The oracle cannot step 16.8 M cells in test time, so this run checks the
properties that hold at any size (m0 from the planner generator with seed 44,
DP45 at max_error 1e-5 with dt_max 1e-10, the suggested dt fed back):
- |m| = 1 on the active cells and m = 0 outside the geometry, after every step;
- with damping and a static field the total energy does not increase from one
  accepted step to the next;
- every statistic is finite, and the suggested dt stays positive.
The same kernels are compared with the oracle on two bands of this geometry
that keep its 2048-point x and y lines, nz = 16 and the mask
(test_gpu_headline_sizes.py).
"""
import numpy as np
import pytest

from fullmag_b200 import native_fdm as nf

MU0 = 4.0 * np.pi * 1e-7


def _disk(nx, ny, nz, r_out, r_in, d):
    x = (np.arange(nx) + 0.5) * d - nx * d / 2
    y = (np.arange(ny) + 0.5) * d - ny * d / 2
    X, Y = np.meshgrid(x, y)
    r2 = X ** 2 + Y ** 2
    m2 = (r2 <= r_out ** 2) & (r2 > r_in ** 2)
    return np.repeat(m2[None], nz, axis=0).astype(np.uint8).reshape(-1)


@pytest.mark.gpu
def test_c3_full_size_masked_dp45_properties():
    nx, ny, nz, d = 1024, 1024, 16, 2e-9
    n = nx * ny * nz
    # disk of radius 1 um with a centred hole of 300 nm diameter; Ms = 0 outside
    mask = _disk(nx, ny, nz, 1e-6, 150e-9, d)
    active = mask.astype(bool)
    m0 = nf.random_unit_vectors(44, n)
    plan = nf.FdmPlan(cells=(nx, ny, nz), cell_size=(d, d, d), initial_magnetization=m0,
                      saturation_magnetisation=8e5, exchange_stiffness=1.3e-11, damping=0.1,
                      gyromagnetic_ratio=2.211e5, precision=nf.PRECISION_SINGLE, integrator=nf.DP45,
                      enable_exchange=True, enable_demag=True, external_field=(0.0, 30e-3 / MU0, 0.0),
                      active_mask=mask, adaptive=(1e-5, 1e-18, 1e-10, 0.8), demag_source=nf.DEMAG_NEWELL)
    be = nf.NativeFdmBackend(plan)
    dt = 1e-13
    energies = []
    for k in range(10):
        st = be.step(dt)
        for key, v in st.items():
            assert np.isfinite(v), (k, key, v)
        assert st["suggested_next_dt"] > 0.0, st
        dt = st["suggested_next_dt"]
        energies.append(st["total_energy_joules"])
        if k in (0, 9):
            m = be.copy_m().reshape(-1, 3)
            norms = np.linalg.norm(m[active], axis=1)
            assert np.abs(norms - 1.0).max() < 1e-5, (k, np.abs(norms - 1.0).max())
            assert np.abs(m[~active]).max() == 0.0, k
    for k in range(1, len(energies)):
        assert energies[k] <= energies[k - 1] + 1e-6 * abs(energies[k - 1]), (k, energies)
    assert energies[-1] < energies[0], energies
    be.close()
