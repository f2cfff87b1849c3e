"""CPU-side checks of the drop-in C ABI library (no CUDA device needed).

- include/fullmag_fdm.h has the reference header's exact binary layout
  (fixture generated from native/include/fullmag_fdm.h by
  tests/golden/make_abi_layout.py);
- libfullmag_fdm.so.0 loads and exports every function the headers declare;
- the ctypes mirror in fullmag_b200.native_fdm has the same sizes;
- host-only entry points (null handles, plan validation, FP64 Newell
  spectra) behave as the reference contract says.
"""
import ctypes as C
import json
import os
import re
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import make_abi_layout as layout  # noqa: E402
from fullmag_b200 import native_fdm as nf  # noqa: E402
from oracle import oracle as O  # noqa: E402


def _declared_functions():
    names = set()
    for h in ("fullmag_fdm.h", "fullmag_fdm_ext.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(fullmag_fdm_\w+)\s*\(", src))
    return sorted(names)


def test_header_layout_matches_reference_fixture():
    ref = json.load(open(layout.FIXTURE))
    mine = layout.layout_of(os.path.join(ROOT, "include"))
    diffs = {k: (ref[k], mine.get(k)) for k in ref if ref[k] != mine.get(k)}
    assert not diffs


def test_ctypes_mirror_sizes():
    ref = json.load(open(layout.FIXTURE))
    assert C.sizeof(nf.PlanDesc) == ref["sizeof fullmag_fdm_plan_desc"]
    assert C.sizeof(nf.StepStats) == ref["sizeof fullmag_fdm_step_stats"]
    assert C.sizeof(nf.DeviceInfo) == ref["sizeof fullmag_fdm_device_info"]
    assert C.sizeof(nf.SnapshotDesc) == ref["sizeof fullmag_fdm_snapshot_desc"]
    for f, _ in nf.PlanDesc._fields_:
        assert getattr(nf.PlanDesc, f).offset == ref[f"fullmag_fdm_plan_desc.{f}"][0], f


def test_library_exports_every_declared_function():
    lib = nf.load_library()
    declared = _declared_functions()
    assert set(nf.ABI_FUNCTIONS) <= set(declared)
    assert set(nf.EXT_FUNCTIONS) <= set(declared)
    for name in declared:
        assert hasattr(lib, name), name
    # the ABI surface of the reference: 16 entry points, all present
    assert len(nf.ABI_FUNCTIONS) == 16


def test_null_handle_contract():
    lib = nf.load_library()
    assert lib.fullmag_fdm_backend_last_error(None) == b"null handle"
    assert lib.fullmag_fdm_backend_create(None) is None
    lib.fullmag_fdm_backend_destroy(None)
    lib.fullmag_fdm_field_snapshot_destroy(None)
    st = nf.StepStats()
    assert lib.fullmag_fdm_backend_step(None, 1e-13, C.byref(st)) == nf.ERR_INVALID
    assert lib.fullmag_fdm_backend_refresh_observables(None) == nf.ERR_INVALID


def _bad_plan_error(**kw):
    """create() with an invalid plan: the handle comes back with last_error set."""
    n = 4 * 3 * 2
    base = dict(cells=(4, 3, 2), cell_size=(2e-9, 2e-9, 2e-9),
                initial_magnetization=np.tile([1.0, 0, 0], n), enable_demag=False)
    base.update(kw)
    plan = nf.FdmPlan(**base)
    lib = nf.load_library()
    desc = plan.to_desc()
    ext = plan.to_ext()
    if ext is None:
        h = lib.fullmag_fdm_backend_create(C.byref(desc))
    else:
        h = lib.fullmag_fdm_backend_create_ext(C.byref(desc), C.byref(ext))
    assert h is not None
    err = lib.fullmag_fdm_backend_last_error(h)
    lib.fullmag_fdm_backend_destroy(h)
    return err.decode() if err else None


def test_validation_errors_without_device():
    assert "initial_magnetization_len mismatch" in _bad_plan_error(initial_magnetization=np.zeros(9))
    assert "unknown integrator" in _bad_plan_error(integrator=9)
    assert "active_mask_len mismatch" in _bad_plan_error(active_mask=np.ones(5))
    assert "region id" in _bad_plan_error(region_mask=np.full(24, 300))
    assert "cell sizes" in _bad_plan_error(cell_size=(0.0, 1e-9, 1e-9))
    assert "saturation" in _bad_plan_error(saturation_magnetisation=0.0)
    assert "spectrum_len mismatch" in _bad_plan_error(enable_demag=True, demag_spectra=[np.zeros(10)] * 6)
    assert "prime factor" in _bad_plan_error(cells=(11, 3, 2), initial_magnetization=np.zeros(3 * 66),
                                             enable_demag=True)


def test_boundary_tier_validation_without_device():
    """Boundary tiers: the reference skips a tier silently when the volume
    fraction is missing or has the wrong length, and reads out of bounds on
    bad correction indices; here these are create errors."""
    ones = np.ones(24)
    assert "unknown boundary_correction" in _bad_plan_error(boundary_correction=7, volume_fraction=ones)
    assert "volume_fraction is required" in _bad_plan_error(boundary_correction=nf.BOUNDARY_VOLUME)
    assert "volume_fraction_len mismatch" in _bad_plan_error(boundary_correction=nf.BOUNDARY_FULL,
                                                             volume_fraction=np.ones(5))
    corr = (np.array([3], np.int32), np.array([[2, 99]], np.int32), np.zeros((1, 2, 6)))
    assert "demag_corr_source_idx 99 out of range" in _bad_plan_error(
        boundary_correction=nf.BOUNDARY_VOLUME, volume_fraction=ones, demag_corr=corr)
    assert "per-cell Ms map" in _bad_plan_error(boundary_correction=nf.BOUNDARY_VOLUME, volume_fraction=ones,
                                                ms_map=np.full(24, 8e5))


@pytest.mark.parametrize("dims", [(5, 4, 3), (8, 6, 1), (16, 8, 2), (45, 3, 1)])
def test_newell_spectra_host_code_matches_oracle(dims):
    nx, ny, nz = dims
    d = (2e-9, 2.5e-9, 3e-9)
    for thin in ((False, True) if nz == 1 else (False,)):
        got = nf.newell_spectra(nx, ny, nz, *d, thin_film_2d=thin)
        ref = O.newell_spectra(nx, ny, nz, *d, thin_film_2d=thin)
        scale = max(np.abs(r).max() for r in ref[:3])
        for c in range(6):
            assert np.abs(got[c] - ref[c]).max() <= 1e-12 * scale, (dims, thin, c)
