"""Pins of the FP64 CPU oracle against the reference's own known answers.

Every test here restates a reference test or golden value:
  crates/fullmag-fdm-demag/src/newell.rs:676-907   (Newell tensor)
  crates/fullmag-engine/src/lib.rs:2976-3289       (engine)
  crates/fullmag-plan/src/lib.rs:1928-1957          (seeded unit vectors)
and the FFT (the reference uses rustfft 6.4.1, not vendored) is checked
against numpy.fft.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

MU0 = 4.0 * np.pi * 1e-7


# ---------------------------------------------------------------- FFT
@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 8, 12, 16, 30, 37, 64, 74, 96, 105, 128, 1024])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    scale = np.abs(x).sum()
    assert np.abs(O.fft(x) - np.fft.fft(x)).max() <= 1e-14 * scale
    assert np.abs(O.fft(x, inverse=True) - np.fft.ifft(x) * n).max() <= 1e-14 * scale


# ---------------------------------------------------------------- Newell (newell.rs tests)
def test_f_g_at_origin_are_zero():
    assert O.newell_f(0.0, 0.0, 0.0) == 0.0
    assert O.newell_g(0.0, 0.0, 0.0) == 0.0


def test_self_term_trace_cubic_and_one_third():
    k = O.newell_kernels(1, 1, 1, 1.0, 1.0, 1.0)
    assert abs(k[0, 0, 0, 0] + k[1, 0, 0, 0] + k[2, 0, 0, 0] - 1.0) < 1e-10
    assert abs(k[0, 0, 0, 0] - 1.0 / 3.0) < 1e-6


def test_self_term_noncubic():
    k = O.newell_kernels(1, 1, 1, 5e-9, 5e-9, 2e-9)
    assert abs(k[0, 0, 0, 0] + k[1, 0, 0, 0] + k[2, 0, 0, 0] - 1.0) < 1e-10
    assert k[2, 0, 0, 0] > k[0, 0, 0, 0]
    assert abs(k[0, 0, 0, 0] - k[1, 0, 0, 0]) < 1e-12


def test_off_diagonal_self_terms_zero():
    k = O.newell_kernels(1, 1, 1, 3e-9, 4e-9, 5e-9)
    for c in (3, 4, 5):
        assert abs(k[c, 0, 0, 0]) < 1e-12


def test_kernel_parity():
    k = O.newell_kernels(4, 4, 4, 1.0, 1.0, 1.0)
    px = 8
    # index order (z, y, x)
    assert abs(k[0, 3, 2, 1] - k[0, 3, 2, px - 1]) < 1e-15
    assert abs(k[3, 3, 2, 1] + k[3, 3, 2, px - 1]) < 1e-15


def test_nxy_golden_values():
    k = O.newell_kernels(10, 10, 1, 1.0, 1.0, 1.0)
    nxy = k[3, 0]
    assert abs(nxy[1, 1] - (-4.5565e-2)) < 1e-5      # reference -4.55648226e-02
    assert abs(nxy[2, 2] - (-5.2897e-3)) < 1e-6      # reference -5.28968456e-03
    assert abs(nxy[5, 5] - (-3.3764e-4)) < 5e-8      # reference -3.37642932e-04
    assert abs(nxy[0, 1]) < 1e-15
    for i in range(1, 5):
        for j in range(1, 5):
            assert nxy[j, i] < 0.0
    # tighter: the reference comment's 9-digit values
    assert abs(nxy[1, 1] - (-4.55648226e-02)) < 5e-11
    assert abs(nxy[2, 2] - (-5.28968456e-03)) < 5e-12
    assert abs(nxy[5, 5] - (-3.37642932e-04)) < 5e-13


def test_nxy_far_field_asymptote():
    k = O.newell_kernels(12, 12, 1, 1.0, 1.0, 1.0)
    x = y = 8.0
    asym = -3.0 * x * y / (4.0 * np.pi * (x * x + y * y) ** 2.5)
    assert abs(k[3, 0, 8, 8] - asym) / abs(asym) < 1e-3


def test_thin_cell_nzz_dominates():
    k = O.newell_kernels(1, 1, 1, 5e-9, 5e-9, 1e-9)
    assert k[2, 0, 0, 0] > k[0, 0, 0, 0]
    assert abs(k[0, 0, 0, 0] + k[1, 0, 0, 0] + k[2, 0, 0, 0] - 1.0) < 1e-10
    assert k[2, 0, 0, 0] > 0.5


def test_spectra_real_and_symmetric():
    sp = O.newell_spectra(6, 5, 3, 2e-9, 2.5e-9, 3e-9)
    for c, s in enumerate(sp):
        z = s[0::2] + 1j * s[1::2]
        assert np.abs(z.imag).max() < 1e-12 * np.abs(z.real).max()


def test_spectra_equal_fft_of_real_space_kernel():
    nx, ny, nz = 5, 4, 3
    k = O.newell_kernels(nx, ny, nz, 1e-9, 2e-9, 3e-9)
    sp = O.newell_spectra(nx, ny, nz, 1e-9, 2e-9, 3e-9)
    for c in range(6):
        ref = np.fft.fftn(k[c]).reshape(-1)
        got = sp[c][0::2] + 1j * sp[c][1::2]
        assert np.abs(got - ref).max() < 1e-13 * np.abs(ref).max()


# ---------------------------------------------------------------- seeded m0 (fullmag-plan lib.rs:1928-1957)
def _xorshift_unit_vectors(seed, count):
    state = seed
    out = []
    mask = (1 << 64) - 1
    for _ in range(count):
        while True:
            c = []
            for _ in range(3):
                state ^= (state << 13) & mask
                state ^= state >> 7
                state ^= (state << 17) & mask
                c.append((float(state) / float(mask)) * 2.0 - 1.0)
            nrm = math.sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2])
            if nrm > 1e-10:
                out.extend(v / nrm for v in c)
                break
    return np.array(out)


@pytest.mark.parametrize("seed", [42, 43, 7])
def test_random_unit_vectors_match_xorshift(seed):
    got = O.random_unit_vectors(seed, 257)
    ref = _xorshift_unit_vectors(seed, 257)
    assert np.array_equal(got, ref)
    assert np.allclose(np.linalg.norm(got.reshape(-1, 3), axis=1), 1.0, atol=1e-15)


# ---------------------------------------------------------------- engine known answers (lib.rs tests)
def simple_problem(alpha, gamma):
    return O.Problem(3, 1, 1, 1.0, 1.0, 1.0, ms=1.0, aex=0.5 * MU0, alpha=alpha, gamma=gamma,
                     demag=False)


def test_uniform_state_zero_exchange_and_rhs():
    s = O.Simulation(simple_problem(0.1, 1.0), np.tile([1.0, 0, 0], 3))
    obs = s.observe()
    assert np.abs(obs["h_ex"]).max() <= 1e-12
    assert np.abs(obs["rhs"]).max() <= 1e-12
    assert obs["e_ex_pair"] <= 1e-12


def test_center_exchange_field_second_difference():
    s = O.Simulation(simple_problem(0.0, 1.0), np.array([1, 0, 0, 0, 1, 0, 1, 0, 0.0]))
    assert np.allclose(s.observe()["h_ex"].reshape(-1, 3)[1], [2.0, -2.0, 0.0], atol=1e-12)


def test_masked_exchange_free_surface():
    p = O.Problem(3, 1, 1, 1.0, 1.0, 1.0, ms=1.0, aex=0.5 * MU0, alpha=0.1, gamma=1.0, demag=False,
                  active_mask=np.array([1, 1, 0]))
    s = O.Simulation(p, np.array([1, 0, 0, 0, 1, 0, 0.7, 0.3, 0.0]))
    h = s.observe()["h_ex"].reshape(-1, 3)
    assert np.allclose(h[1], [1.0, -1.0, 0.0], atol=1e-12)
    assert np.allclose(h[2], 0.0, atol=1e-12)
    assert np.allclose(s.m.reshape(-1, 3)[2], 0.0)


def test_masked_demag_and_external_zero_outside():
    p = O.Problem(3, 1, 1, 1.0, 1.0, 1.0, ms=1.0, aex=0.5 * MU0, alpha=0.1, gamma=1.0,
                  exchange=False, h_ext=(0, 0, 1.0), active_mask=np.array([1, 1, 0]))
    s = O.Simulation(p, np.array([1, 0, 0, 1, 0, 0, 0, 1, 0.0]))
    obs = s.observe()
    for k in ("h_ext", "h_demag", "h_eff"):
        assert np.allclose(obs[k].reshape(-1, 3)[2], 0.0, atol=1e-12)


def test_heun_preserves_unit_norm():
    s = O.Simulation(simple_problem(0.1, 1.0), np.array([1, 0, 0, 0, 1, 0, 1, 0, 0.0]))
    s.step(1e-3)
    assert np.allclose(np.linalg.norm(s.m.reshape(-1, 3), axis=1), 1.0, atol=1e-12)


def test_damped_relaxation_reduces_exchange_energy():
    s = O.Simulation(simple_problem(0.5, 1.0), np.array([1, 0, 0, 0, 1, 0, 1, 0, 0.0]))
    e0 = s.observe()["e_ex_field"]
    for _ in range(10):
        s.step(1e-3)
    assert s.observe()["e_total"] < e0


def test_zeeman_relaxation_and_pure_damping():
    p = O.Problem(2, 1, 1, 1.0, 1.0, 1.0, ms=1.0, aex=0.5 * MU0, alpha=0.5, gamma=1.0,
                  exchange=False, demag=False, h_ext=(0, 0, 1.0))
    s = O.Simulation(p, np.tile([1.0, 0, 0], 2))
    e0 = s.observe()["e_ext"]
    for _ in range(100):
        s.step(5e-3)
    assert s.observe()["e_ext"] < e0
    assert s.m[2] > 0.1
    p.precession = False
    s2 = O.Simulation(p, np.tile([1.0, 0, 0], 2))
    s2.step(1e-3)
    assert abs(s2.m[1]) <= 1e-12 and s2.m[2] > 0.0


def demag_problem(nx, ny, nz):
    return O.Problem(nx, ny, nz, 1.0, 1.0, 0.2, ms=1.0, aex=0.5 * MU0, alpha=0.1, gamma=1.0,
                     exchange=False)


def test_thin_film_demag_orderings():
    p = demag_problem(4, 4, 1)
    e_out = O.Simulation(p, np.tile([0, 0, 1.0], 16)).observe()["e_demag"]
    e_in = O.Simulation(p, np.tile([1.0, 0, 0], 16)).observe()["e_demag"]
    assert e_out > e_in
    p8 = demag_problem(8, 8, 1)
    e_in8 = O.Simulation(p8, np.tile([1.0, 0, 0], 64)).observe()["e_demag"]
    e_out8 = O.Simulation(p8, np.tile([0, 0, 1.0], 64)).observe()["e_demag"]
    assert e_in8 < 0.5 * e_out8


def test_demag_energy_nonnegative_random():
    rng = np.random.default_rng(42)
    m = rng.uniform(-1, 1, (32, 3))
    e = O.Simulation(demag_problem(4, 4, 2), m).observe()["e_demag"]
    assert e >= 0.0 and np.isfinite(e)


def test_total_energy_decreases_with_demag():
    p = O.Problem(8, 8, 1, 2e-9, 2e-9, 2e-9, ms=800e3, aex=13e-12, alpha=0.5)
    l = np.sqrt(0.01 ** 2 * 2 + 1)
    s = O.Simulation(p, np.tile([0.01 / l, 0.01 / l, 1 / l], 64))
    e0 = s.observe()["e_total"]
    for _ in range(200):
        s.step(1e-14)
    assert s.observe()["e_total"] < e0


def test_thin_film_2d_path_equals_3d_path():
    m0 = O.random_unit_vectors(42, 8 * 6)
    kw = dict(ms=8e5, aex=1.3e-11, alpha=0.02, h_ext=(-20e-3 / MU0, 5e-3 / MU0, 0))
    a = O.Simulation(O.Problem(8, 6, 1, 3.125e-9, 3.125e-9, 3e-9, **kw), m0)
    b = O.Simulation(O.Problem(8, 6, 1, 3.125e-9, 3.125e-9, 3e-9, thin_film_2d=True, **kw), m0)
    for _ in range(5):
        a.step(1e-13)
        b.step(1e-13)
    assert np.array_equal(a.m, b.m)


def test_pair_and_field_exchange_energy_agree():
    p = O.Problem(7, 5, 3, 2e-9, 2e-9, 2e-9, demag=False)
    s = O.Simulation(p, O.random_unit_vectors(3, 105))
    obs = s.observe()
    assert abs(obs["e_ex_pair"] - obs["e_ex_field"]) <= 1e-10 * abs(obs["e_ex_field"])


def test_dp45_controller_accepts_and_suggests():
    p = O.Problem(8, 8, 1, 2e-9, 2e-9, 2e-9, ms=8e5, aex=1.3e-11, alpha=0.1, integrator=O.DP45,
                  max_error=1e-5)
    s = O.Simulation(p, O.random_unit_vectors(44, 64))
    r = s.step(1e-13)
    assert r["dt_used"] <= 1e-13 and r["suggested_next_dt"] > 0
    assert abs(s.time - r["dt_used"]) < 1e-30


# ---------------------------------------------------------------- RK4 / RK23 / ABM3
# The reference has no known-answer tests for these integrators; the
# restatement (lib.rs:1253-1407, 1573-1648) is pinned by its convergence
# order on a smooth, non-chaotic problem, by the Heun start-up of ABM3 and by
# the step controller of RK23.
def _smooth_problem(integrator, **kw):
    nx, ny, nz = 16, 8, 1
    x = (np.arange(nx) + 0.5) / nx
    m0 = np.zeros((nx * ny * nz, 3))
    m0[:, 0] = np.tile(np.cos(0.6 * np.pi * x), ny)
    m0[:, 1] = np.tile(np.sin(0.6 * np.pi * x), ny)
    m0[:, 2] = 0.3
    prob = O.Problem(nx, ny, nz, 3e-9, 3e-9, 3e-9, alpha=0.1, integrator=integrator,
                     h_ext=(5e3, 2e4, -1e4), thin_film_2d=True, **kw)
    return prob, m0.reshape(-1)


def _final_m(integrator, dt, t_end, **kw):
    prob, m0 = _smooth_problem(integrator, **kw)
    sim = O.Simulation(prob, m0)
    for _ in range(int(round(t_end / dt))):
        sim.step(dt)
    return sim.m


@pytest.fixture(scope="module")
def smooth_reference():
    return _final_m(O.RK4, 1e-15, 4e-12)


# measured rates: RK4 4.01, ABM3 2.89 (its Heun start-up steps still show at
# this dt), Heun 2.00
@pytest.mark.parametrize("integrator,order", [(O.RK4, 4), (O.ABM3, 3), (O.HEUN, 2)])
def test_fixed_step_integrators_converge_at_their_order(integrator, order, smooth_reference):
    e1 = np.abs(_final_m(integrator, 2e-14, 4e-12) - smooth_reference).max()
    e2 = np.abs(_final_m(integrator, 1e-14, 4e-12) - smooth_reference).max()
    rate = math.log2(e1 / e2)
    assert order - 0.45 <= rate <= order + 0.45, (e1, e2, rate)


def test_rk23_fixed_step_is_third_order(smooth_reference):
    """max_error far above any error estimate makes every attempt accept, so
    RK23 runs at the given dt (the clamps are set around it)."""
    errs = []
    for dt in (2e-14, 1e-14):
        errs.append(np.abs(_final_m(O.RK23, dt, 4e-12, max_error=1e30, dt_min=1e-18, dt_max=1.0,
                                    headroom=0.8) - smooth_reference).max())
    rate = math.log2(errs[0] / errs[1])
    assert 2.55 <= rate <= 3.45, (errs, rate)


def test_abm3_startup_steps_are_heun_steps():
    prob_h, m0 = _smooth_problem(O.HEUN)
    prob_a, _ = _smooth_problem(O.ABM3)
    h, a = O.Simulation(prob_h, m0), O.Simulation(prob_a, m0)
    for _ in range(3):
        rh, ra = h.step(1e-13), a.step(1e-13)
        assert np.array_equal(h.m, a.m)
        # energies are OpenMP reductions: summation order varies by a few ulp
        assert abs(rh["e_total"] - ra["e_total"]) <= 1e-12 * abs(rh["e_total"])
    h.step(1e-13)
    a.step(1e-13)  # the first multistep step differs from Heun
    assert not np.array_equal(h.m, a.m)


def test_abm3_restarts_with_heun_when_dt_changes():
    """More than 10 % change of dt: three Heun steps again, from the same state."""
    prob_a, m0 = _smooth_problem(O.ABM3)
    a = O.Simulation(prob_a, m0)
    for _ in range(5):
        a.step(1e-13)
    prob_h, _ = _smooth_problem(O.HEUN)
    h = O.Simulation(prob_h, a.m)  # (re-normalised on creation: last-bit changes only)
    for _ in range(3):
        a.step(1.5e-13)
        h.step(1.5e-13)
        assert np.abs(h.m - a.m).max() <= 1e-13
    # a change of less than 10 % keeps the history
    b = O.Simulation(prob_a, m0)
    c = O.Simulation(prob_a, m0)
    for _ in range(5):
        b.step(1e-13)
        c.step(1e-13)
    b.step(1.05e-13)
    h2 = O.Simulation(prob_h, c.m)
    h2.step(1.05e-13)
    assert np.abs(b.m - h2.m).max() > 1e-11


def test_rk23_controller_rejects_and_suggests():
    prob, m0 = _smooth_problem(O.RK23, max_error=1e-7, dt_min=1e-18, dt_max=1e-10, headroom=0.8)
    sim = O.Simulation(prob, m0)
    r = sim.step(5e-12)  # far too large for 1e-7: rejected at least once
    assert r["rejected_attempts"] >= 1
    assert r["dt_used"] < 5e-12
    # the next suggestion follows headroom * dt * (max_error / err)^(1/3), clamped
    assert 0.0 < r["suggested_next_dt"] <= 1e-10
    dt = r["suggested_next_dt"]
    r2 = sim.step(dt)
    assert r2["dt_used"] == dt or r2["rejected_attempts"] > 0


# ---------------------------------------------------------------- boundary tiers
# exchange_t0_fp64.cu, exchange_t1_fp64.cu, demag_fp64.cu:79-85,
# demag_boundary_fp64.cu.  The reference has no tests for the tiers; the
# restatement is pinned by the interior limit (phi = 1, full faces, distances =
# cell size: the tiers must reproduce the standard fields) and by the sparse
# correction adding exactly -dN M at its targets.
def _tier_problem(tier, nx=12, ny=10, nz=3, **kw):
    n = nx * ny * nz
    d = (2e-9, 2.5e-9, 3e-9)
    vf = np.ones(n)
    faces = [np.ones(n) for _ in range(6)]
    deltas = [np.full(n, d[q // 2]) for q in range(6)]
    prob = O.Problem(nx, ny, nz, *d, alpha=0.1, h_ext=(1e4, -2e4, 5e3), boundary_tier=tier,
                     volume_fraction=vf, face_link=faces, delta=deltas, **kw)
    return prob, O.random_unit_vectors(9, n)


@pytest.mark.parametrize("tier", [1, 2])
def test_tier_interior_limit_equals_standard_fields(tier):
    prob, m0 = _tier_problem(tier)
    base, _ = _tier_problem(0)
    a = O.Simulation(prob, m0).observe()
    b = O.Simulation(base, m0).observe()
    for key in ("h_ex", "h_demag", "h_eff"):
        scale = np.abs(b[key]).max()
        assert np.abs(a[key] - b[key]).max() <= 1e-12 * scale, key


def test_tier_demag_correction_adds_minus_dn_m():
    rng = np.random.default_rng(3)
    prob, m0 = _tier_problem(1)
    n = prob.nx * prob.ny * prob.nz
    targets = np.array([5, 17, 40, 77], np.int32)
    sources = rng.integers(-1, n, size=(4, 5)).astype(np.int32)
    tensors = rng.uniform(-1e-3, 1e-3, size=(4, 5, 6))
    plain = O.Simulation(prob, m0)
    prob.corr_target, prob.corr_source, prob.corr_tensor = targets, sources, tensors
    corr = O.Simulation(prob, m0)
    h0 = plain.observe()["h_demag"].reshape(-1, 3)
    h1 = corr.observe()["h_demag"].reshape(-1, 3)
    m = plain.m.reshape(-1, 3)
    want = np.zeros_like(h0)
    for t, ti in enumerate(targets):
        for q, si in enumerate(sources[t]):
            if si < 0:
                continue
            xx, xy, xz, yy, yz, zz = tensors[t, q]
            N = np.array([[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]])
            want[ti] -= N @ (prob.ms * 1.0 * m[si])
    assert np.abs((h1 - h0) - want).max() <= 1e-12 * np.abs(h0).max()
    untouched = np.setdiff1d(np.arange(n), targets)
    assert np.array_equal(h1[untouched], h0[untouched])
