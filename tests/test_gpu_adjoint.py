"""Adjoint of the Heun trajectory (fullmag_fdm_adjoint_forward / _backward):
dL/dMs per cell, dL/dH_ext, dL/dH_ac and dL/dm0 of L = sum of m_x over a
central region of the final state.

Checks:
  - against central finite differences of the FP64 CPU oracle on a small C5-like
    film (Ms map, B(t) = (20 sin(2 pi 5 GHz t), 0, 5) mT), 1e-6 of the largest
    dL/dMs per cell and 1e-7 relative for the fields (FD step h = 1e-4 of the
    parameter; measured agreement 1e-8 and 1e-9);
  - dL/dm0 against finite differences of the library's own FP64 forward (the
    oracle normalises m0 on creation, the library keeps the uploaded m0);
  - bit-identical gradients for every checkpoint interval (exact replay);
  - at the C5 size (256 x 256 x 1, 2000 steps, uniform m0 along +y) FP64
    against FD of the library's FP64 forward, and FP32 against FP64;
  - the torch.autograd.Function wrapper returns the C API's gradients.
"""
import numpy as np
import pytest
import torch

from fullmag_b200 import native_fdm as nf
from fullmag_b200.adjoint import HeunTrajectory
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MU0 = 4e-7 * np.pi
H_EXT = (0.0, 0.0, 5e-3 / MU0)
H_AC = (20e-3 / MU0, 0.0, 0.0)
FREQ = 5e9


def _c5_inputs(nx, ny, seed=46):
    rng = np.random.default_rng(seed)
    ms_map = rng.uniform(6e5, 1e6, nx * ny)
    m0 = O.random_unit_vectors(seed, nx * ny)
    return ms_map, m0


def _region(nx, ny, w):
    sel = np.zeros((ny, nx), bool)
    sel[(ny - w) // 2:(ny + w) // 2, (nx - w) // 2:(nx + w) // 2] = True
    return sel.reshape(-1)


def _plan(nx, ny, m0, ms_map, h_ext=H_EXT, h_ac=H_AC, precision=nf.PRECISION_DOUBLE):
    return nf.FdmPlan(cells=(nx, ny, 1), cell_size=(4e-9, 4e-9, 3e-9), initial_magnetization=m0,
                      exchange_stiffness=1.3e-11, damping=0.05, gyromagnetic_ratio=2.211e5,
                      precision=precision, external_field=h_ext, ms_map=ms_map, ac_field=h_ac,
                      ac_frequency_hz=FREQ, demag_source=nf.DEMAG_NEWELL)


def _adjoint(nx, ny, m0, ms_map, dt, n, region, precision=nf.PRECISION_DOUBLE, K=0):
    with nf.NativeFdmBackend(_plan(nx, ny, m0, ms_map, precision=precision)) as be:
        be.adjoint_forward(dt, n, K)
        m = be.copy_m().reshape(-1, 3)
        loss = m[region, 0].sum()
        g = np.zeros((nx * ny, 3))
        g[region, 0] = 1.0
        grads = be.adjoint_backward(g.reshape(-1))
        # the backend is back at the final state
        assert np.array_equal(be.copy_m().reshape(-1, 3), m)
    return loss, grads


def _oracle_loss(nx, ny, m0, ms_map, dt, n, region, h_ext=H_EXT, h_ac=H_AC):
    prob = O.Problem(nx, ny, 1, 4e-9, 4e-9, 3e-9, aex=1.3e-11, alpha=0.05, gamma=2.211e5,
                     ms=float(ms_map.mean()), ms_map=ms_map, h_ext=h_ext, h_ac=h_ac, ac_freq=FREQ,
                     thin_film_2d=True)
    sim = O.Simulation(prob, m0)
    for _ in range(n):
        sim.step(dt)
    return sim.m.reshape(-1, 3)[region, 0].sum()


def _gpu_loss(nx, ny, m0, ms_map, dt, n, region, h_ext=H_EXT, h_ac=H_AC):
    with nf.NativeFdmBackend(_plan(nx, ny, m0, ms_map, h_ext, h_ac)) as be:
        be.step_n(dt, n)
        return be.copy_m().reshape(-1, 3)[region, 0].sum()


def test_adjoint_matches_oracle_finite_differences():
    nx = ny = 16
    dt, n = 1e-13, 40
    ms_map, m0 = _c5_inputs(nx, ny)
    region = _region(nx, ny, 8)
    loss, g = _adjoint(nx, ny, m0, ms_map, dt, n, region)
    assert abs(loss - _oracle_loss(nx, ny, m0, ms_map, dt, n, region)) <= 1e-9
    for cell in (0, 37, 119, 136, 255):
        h = 1e-4 * ms_map[cell]
        mp, mm = ms_map.copy(), ms_map.copy()
        mp[cell] += h
        mm[cell] -= h
        fd = (_oracle_loss(nx, ny, m0, mp, dt, n, region) - _oracle_loss(nx, ny, m0, mm, dt, n, region)) / (2 * h)
        print("dL/dMs", cell, g["dl_dms"][cell], fd)
        assert abs(g["dl_dms"][cell] - fd) <= 1e-6 * np.abs(g["dl_dms"]).max(), cell
    for name, base, c in (("dl_dh_ac", H_AC, 0), ("dl_dh_ext", H_EXT, 2), ("dl_dh_ext", H_EXT, 0)):
        h = 1e-4 * max(abs(base[c]), 1e3)
        bp, bm = list(base), list(base)
        bp[c] += h
        bm[c] -= h
        kw_p = {"h_ac": tuple(bp)} if name == "dl_dh_ac" else {"h_ext": tuple(bp)}
        kw_m = {"h_ac": tuple(bm)} if name == "dl_dh_ac" else {"h_ext": tuple(bm)}
        fd = (_oracle_loss(nx, ny, m0, ms_map, dt, n, region, **kw_p) -
              _oracle_loss(nx, ny, m0, ms_map, dt, n, region, **kw_m)) / (2 * h)
        print(name, c, g[name][c], fd)
        assert abs(g[name][c] - fd) <= 1e-7 * max(abs(fd), 1e-12) + 1e-14, (name, c)


def test_adjoint_dm0_matches_library_finite_differences():
    nx = ny = 16
    dt, n = 1e-13, 30
    ms_map, m0 = _c5_inputs(nx, ny, seed=7)
    region = _region(nx, ny, 8)
    _, g = _adjoint(nx, ny, m0, ms_map, dt, n, region)
    for k in (3 * 40 + 0, 3 * 120 + 1, 3 * 135 + 2):
        h = 1e-6
        mp, mm = m0.copy(), m0.copy()
        mp[k] += h
        mm[k] -= h
        fd = (_gpu_loss(nx, ny, mp, ms_map, dt, n, region) - _gpu_loss(nx, ny, mm, ms_map, dt, n, region)) / (2 * h)
        assert abs(g["dl_dm0"][k] - fd) <= 1e-6 * max(abs(fd), 1e-3), (k, g["dl_dm0"][k], fd)


def test_adjoint_is_independent_of_the_checkpoint_interval():
    nx = ny = 16
    ms_map, m0 = _c5_inputs(nx, ny, seed=8)
    region = _region(nx, ny, 8)
    ref = None
    for K in (1, 0, 7, 50):
        _, g = _adjoint(nx, ny, m0, ms_map, 1e-13, 50, region, K=K)
        if ref is None:
            ref = g
        for key in ref:
            assert np.array_equal(ref[key], g[key]), (K, key)


def test_c5_size_fp64_vs_finite_differences_and_fp32():
    """C5 starts from a uniform m along +y: with a random m0 (as in the small
    checks above) 2000 steps lie far inside the chaotic regime, where a 1-ulp
    change of the state grows to ~1e-6 (the C1 sensitivity floor) and neither a
    finite difference nor an FP32 run measures a derivative."""
    nx = ny = 256
    dt, n = 1e-13, 2000
    ms_map, _ = _c5_inputs(nx, ny)
    m0 = np.tile([0.0, 1.0, 0.0], nx * ny)
    region = _region(nx, ny, 64)
    loss64, g64 = _adjoint(nx, ny, m0, ms_map, dt, n, region)
    loss32, g32 = _adjoint(nx, ny, m0, ms_map, dt, n, region, precision=nf.PRECISION_SINGLE)
    h = 1e-4 * H_AC[0]
    fd = (_gpu_loss(nx, ny, m0, ms_map, dt, n, region, h_ac=(H_AC[0] + h, 0, 0)) -
          _gpu_loss(nx, ny, m0, ms_map, dt, n, region, h_ac=(H_AC[0] - h, 0, 0))) / (2 * h)
    print("C5 dL/dH_ac_x adjoint", g64["dl_dh_ac"][0], "FD", fd, "FP32", g32["dl_dh_ac"][0])
    assert abs(g64["dl_dh_ac"][0] - fd) <= 1e-6 * abs(fd)          # measured 4e-8
    rel_ms = np.abs(g32["dl_dms"] - g64["dl_dms"]).max() / np.abs(g64["dl_dms"]).max()
    print("C5 FP32 vs FP64 dL/dMs (max rel of max)", rel_ms, "loss", loss64, loss32)
    assert rel_ms <= 1e-4                                              # measured 1.1e-6
    assert abs(g32["dl_dh_ac"][0] - g64["dl_dh_ac"][0]) <= 1e-5 * abs(g64["dl_dh_ac"][0])  # 1.7e-7


def test_torch_autograd_function_matches_c_api():
    nx = ny = 16
    dt, n = 1e-13, 20
    ms_np, m0_np = _c5_inputs(nx, ny, seed=9)
    region = _region(nx, ny, 8)
    _, g = _adjoint(nx, ny, m0_np, ms_np, dt, n, region)
    m0 = torch.tensor(m0_np.reshape(-1, 3), requires_grad=True)
    ms = torch.tensor(ms_np, requires_grad=True)
    he = torch.tensor(H_EXT, dtype=torch.float64, requires_grad=True)
    ha = torch.tensor(H_AC, dtype=torch.float64, requires_grad=True)
    problem = dict(cells=(nx, ny, 1), cell_size=(4e-9, 4e-9, 3e-9), exchange_stiffness=1.3e-11,
                   damping=0.05, gyromagnetic_ratio=2.211e5, ac_frequency_hz=FREQ)
    m = HeunTrajectory.apply(m0, ms, he, ha, problem, dt, n, 0)
    loss = m[torch.from_numpy(region), 0].sum()
    loss.backward()
    assert np.array_equal(ms.grad.numpy(), g["dl_dms"])
    assert np.array_equal(he.grad.numpy(), g["dl_dh_ext"])
    assert np.array_equal(ha.grad.numpy(), g["dl_dh_ac"])
    assert np.array_equal(m0.grad.numpy().reshape(-1), g["dl_dm0"])
