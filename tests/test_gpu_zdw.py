"""The FP32 direct z convolution for 8 < nz <= 16 (k_zdw: each column's outputs
split in two halves over two warps, the column's inputs and table entries
staged in shared memory by cp.async).

- Fields and 5 Heun steps against the FP64 oracle at nz = 9, 12, 14, 15, 16, at
  the FP32-mixed bounds of the other parity tests (fields 2e-6 of each field's
  largest value, m 1e-6); nz = 12 with a mask and an Ms map.  Ly = 32 makes the
  64-column batches straddle kx rows, and 33 x 32 columns leave a partial last
  batch (element copies); Ly = 128 and 256 run the window form (16-byte copies
  of padded table rows; batches on both sides of the ky mirror and the batch
  that starts at Ly / 2).
- The window form equals the element form bitwise (FULLMAG_FDM_ZDW=elem): the
  same table values in the same sums.
- At nz = 8, forced on with FULLMAG_FDM_ZDW=on (fused plane pass off), against
  k_zd: the same table and packed FMAs, so the lower half's z planes of H_d
  are bitwise k_zd's; the upper half, summed in the z-reversed frame, adds each
  +d / -d pair in the other order and agrees to FP32 rounding (1e-6 of max|H_d|).
- At nz = 16 it agrees with the z FFT pass (FULLMAG_FDM_ZCONV=fft).
"""
import numpy as np
import pytest

from fullmag_b200 import native_fdm as nf

from gpu_helpers import make_pair, max_abs

pytestmark = pytest.mark.gpu

_ENV = ("FULLMAG_FDM_FFT", "FULLMAG_FDM_YZ", "FULLMAG_FDM_ZCONV", "FULLMAG_FDM_XPIPE", "FULLMAG_FDM_YZY",
        "FULLMAG_FDM_ZDW")


def _field_errors(be, obs):
    """max |gpu - oracle| of each field relative to that field's own max |H|."""
    out = {}
    for o, key in ((nf.OBS_H_EX, "h_ex"), (nf.OBS_H_DEMAG, "h_demag"), (nf.OBS_H_EFF, "h_eff")):
        ref = obs[key]
        out[key] = max_abs(be.copy_field(o), ref) / max(np.abs(ref).max(), 1e-300)
    return out


def _kernels(be):
    be.set_profiling(True)
    be.refresh_observables()
    names = set(be.profile())
    be.set_profiling(False)
    return names


@pytest.mark.parametrize("cells", [(32, 16, 9), (16, 32, 12), (16, 16, 15), (64, 32, 16), (16, 64, 16), (8, 128, 14)])
def test_wide_direct_z_matches_oracle(monkeypatch, cells):
    for k in _ENV:
        monkeypatch.delenv(k, raising=False)
    nx, ny, nz = cells
    kw = {}
    if cells == (16, 32, 12):
        rng = np.random.default_rng(8)
        kw = dict(mask=(rng.random(nx * ny * nz) > 0.2).astype(np.uint8),
                  ms_map=rng.uniform(6e5, 1e6, nx * ny * nz))
    be, sim, _ = make_pair(cells, (2e-9, 2.5e-9, 3e-9), alpha=0.3, h_ext=(1e4, -5e3, 2e4),
                           precision=nf.PRECISION_SINGLE, symmetric_kernel=True, seed=19, **kw)
    names = _kernels(be)
    assert "demag_z_direct" in names and "demag_z_conv" not in names, names
    err = _field_errors(be, sim.observe())
    print(cells, {k: f"{v:.2e}" for k, v in err.items()})
    for k, v in err.items():
        assert v <= 2e-6, (k, v)
    for _ in range(5):
        be.step(2e-14)
        sim.step(2e-14)
    dm = max_abs(be.copy_m(), sim.m)
    print(cells, f"max|dm| after 5 steps {dm:.2e}")
    assert dm <= 1e-6
    be.close()


def test_wide_direct_z_against_k_zd_at_nz8(monkeypatch):
    for k in _ENV:
        monkeypatch.delenv(k, raising=False)
    monkeypatch.setenv("FULLMAG_FDM_YZY", "off")
    cells = (32, 32, 8)
    kw = dict(cells=cells, cell_size=(2e-9, 2.5e-9, 3e-9), alpha=0.3, h_ext=(1e4, -5e3, 2e4),
              precision=nf.PRECISION_SINGLE, symmetric_kernel=True, seed=23)
    ref, _, _ = make_pair(**kw)
    monkeypatch.setenv("FULLMAG_FDM_ZDW", "on")
    wide, _, _ = make_pair(**kw)
    assert "demag_z_direct" in _kernels(wide)
    ref.refresh_observables()
    nx, ny, nz = cells
    a = wide.copy_field(nf.OBS_H_DEMAG).reshape(nz, ny, nx, 3)
    b = ref.copy_field(nf.OBS_H_DEMAG).reshape(nz, ny, nx, 3)
    assert np.array_equal(a[: nz // 2], b[: nz // 2])
    rel = max_abs(a, b) / np.abs(b).max()
    print(f"nz = 8, k_zdw vs k_zd: {rel:.2e} of max|H_d|")
    assert rel <= 1e-6
    for _ in range(3):
        wide.step(2e-14)
        ref.step(2e-14)
    assert max_abs(wide.copy_m(), ref.copy_m()) <= 1e-6
    wide.close()
    ref.close()


def test_wide_direct_z_agrees_with_z_fft(monkeypatch):
    for k in _ENV:
        monkeypatch.delenv(k, raising=False)
    kw = dict(cells=(32, 64, 16), cell_size=(2e-9, 2e-9, 2e-9), alpha=0.1, h_ext=(0.0, 2e4, 0.0),
              precision=nf.PRECISION_SINGLE, symmetric_kernel=True, seed=29)
    direct, _, _ = make_pair(**kw)
    monkeypatch.setenv("FULLMAG_FDM_ZCONV", "fft")
    zfft, _, _ = make_pair(**kw)
    assert "demag_z_conv" in _kernels(zfft)
    assert "demag_z_direct" in _kernels(direct)
    a, b = direct.copy_field(nf.OBS_H_DEMAG), zfft.copy_field(nf.OBS_H_DEMAG)
    rel = max_abs(a, b) / np.abs(b).max()
    print(f"H_d direct vs z FFT: {rel:.2e} of max|H_d|")
    assert rel <= 2e-6
    direct.close()
    zfft.close()


def test_window_form_equals_element_form_bitwise(monkeypatch):
    for k in _ENV:
        monkeypatch.delenv(k, raising=False)
    kw = dict(cells=(16, 128, 16), cell_size=(2e-9, 2e-9, 2.5e-9), alpha=0.3, h_ext=(1e4, -5e3, 2e4),
              precision=nf.PRECISION_SINGLE, symmetric_kernel=True, seed=31)
    win, _, _ = make_pair(**kw)
    monkeypatch.setenv("FULLMAG_FDM_ZDW", "elem")
    elem, _, _ = make_pair(**kw)
    assert "demag_z_direct" in _kernels(win) and "demag_z_direct" in _kernels(elem)
    for o in (nf.OBS_H_DEMAG, nf.OBS_H_EFF):
        assert np.array_equal(win.copy_field(o), elem.copy_field(o)), o
    for _ in range(3):
        win.step(2e-14)
        elem.step(2e-14)
    assert np.array_equal(win.copy_m(), elem.copy_m())
    win.close()
    elem.close()
