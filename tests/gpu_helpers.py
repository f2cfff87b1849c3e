"""Shared builders for the GPU parity tests: the same seeded problem is given
to the CUDA library (through the C ABI) and to the FP64 oracle."""
import numpy as np

from fullmag_b200 import native_fdm as nf
from oracle import oracle as O

MU0 = 4.0 * np.pi * 1e-7


def c1_kwargs():
    """Config C1: 64x16x1 film of 3.125 x 3.125 x 3 nm cells, B = (-20, 5, 0) mT."""
    return dict(cells=(64, 16, 1), cell_size=(3.125e-9, 3.125e-9, 3e-9), ms=8.0e5, aex=1.3e-11,
                alpha=0.02, gamma=2.211e5, h_ext=(-20e-3 / MU0, 5e-3 / MU0, 0.0), seed=42)


def make_pair(cells, cell_size, ms=8e5, aex=1.3e-11, alpha=0.02, gamma=2.211e5, h_ext=None,
              seed=42, m0=None, mask=None, regions=None, lut=None, demag=True, exchange=True,
              precision=nf.PRECISION_DOUBLE, integrator=nf.HEUN, thin=None, adaptive=None,
              pure_damping=False, spectra="oracle", ms_map=None, ac_field=None, ac_freq=0.0,
              symmetric_kernel=False, boundary=None):
    """Returns (backend, oracle simulation, m0).  symmetric_kernel=True makes the
    oracle convolve with the exactly even/odd Newell spectra the library stores.
    boundary: dict(tier, vf, faces, deltas, corr, phi_floor, delta_min) for the
    boundary tiers (any of faces / deltas / corr may be None)."""
    bnd = boundary or {}
    btier = bnd.get("tier", 0)
    nx, ny, nz = cells
    n = nx * ny * nz
    if m0 is None:
        m0 = O.random_unit_vectors(seed, n)
    if thin is None:
        thin = nz == 1
    spec = None
    demag_source = nf.DEMAG_FROM_PLAN
    if demag and spectra == "oracle":
        spec = O.newell_spectra(nx, ny, nz, *cell_size, thin_film_2d=thin)
    elif demag and spectra == "newell":
        demag_source = nf.DEMAG_NEWELL
    plan = nf.FdmPlan(cells=cells, cell_size=cell_size, initial_magnetization=m0,
                      saturation_magnetisation=ms, exchange_stiffness=aex, damping=alpha,
                      gyromagnetic_ratio=gamma, precision=precision, integrator=integrator,
                      pure_damping=pure_damping, enable_exchange=exchange, enable_demag=demag,
                      external_field=h_ext, active_mask=mask, region_mask=regions,
                      exchange_lut=lut, demag_spectra=spec, adaptive=adaptive, ms_map=ms_map,
                      ac_field=ac_field, ac_frequency_hz=ac_freq, demag_source=demag_source,
                      boundary_correction=btier, boundary_phi_floor=bnd.get("phi_floor", 0.0),
                      boundary_delta_min=bnd.get("delta_min", 0.0), volume_fraction=bnd.get("vf"),
                      face_links=bnd.get("faces"), deltas=bnd.get("deltas"), demag_corr=bnd.get("corr"))
    be = nf.NativeFdmBackend(plan)
    prob = O.Problem(nx, ny, nz, *cell_size, ms=ms, aex=aex, alpha=alpha, gamma=gamma,
                     integrator=integrator,  # the oracle uses the ABI's integrator values
                     precession=not pure_damping, exchange=exchange, demag=demag, h_ext=h_ext,
                     active_mask=mask, region_mask=regions, exchange_lut=lut,
                     ms_map=ms_map, h_ac=ac_field, ac_freq=ac_freq,
                     thin_film_2d=thin and nz == 1, symmetric_kernel=symmetric_kernel,
                     boundary_tier=btier, phi_floor=bnd.get("phi_floor", 0.0),
                     delta_min=bnd.get("delta_min", 0.0), volume_fraction=bnd.get("vf"),
                     face_link=bnd.get("faces"), delta=bnd.get("deltas"))
    if bnd.get("corr") is not None:
        prob.corr_target, prob.corr_source, prob.corr_tensor = bnd["corr"]
    if adaptive is not None:
        prob.max_error, prob.dt_min, prob.dt_max, prob.headroom = adaptive
    sim = O.Simulation(prob, m0)
    return be, sim, m0


def max_abs(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if np.asarray(a).size else 0.0


def rel(a, b):
    d = max(abs(b), 1e-300)
    return abs(a - b) / d
