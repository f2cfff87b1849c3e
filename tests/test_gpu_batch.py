"""The batched ensemble (fullmag_fdm_batch_*): every problem of a batch of
uneven grids and materials, stepped together with one persistent launch per
stage and one CUDA graph per step, against the FP64 oracle run alone on that
problem.  Tolerances as for single problems: FP64 max|dm| <= 1e-10 after 10
Heun steps (inside the predictability horizon of random m0), FP32-mixed 1e-5.
The batch pads each in-plane axis to the smallest power of two or (FP32) 3 * 2^k
(96, 192, 384, 768) >= 2n and z to a power of two, the oracle to 2n: the fields
agree in exact arithmetic (kernel offsets |r| <= n - 1 only).  The shapes cover
padded lengths 16, 32, 64, 96, 128, 192, 256 and 384.  The z convolution runs
as the direct sum over the unpadded z (default; its table is built at the
problem's Lz, which exceeds 2 nz for nz = 3 and 6; FP64 batches with a
problem of nz > 4 keep the z FFT) and as the z FFT pass
(FULLMAG_FDM_BATCH_ZCONV=fft)."""
import numpy as np
import pytest

from fullmag_b200 import native_fdm as nf
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MU0 = 4e-7 * np.pi
SHAPES = [(37, 23, 1), (64, 32, 2), (45, 61, 3), (32, 32, 4), (100, 50, 1), (16, 128, 2), (7, 9, 3),
          (90, 70, 2), (170, 40, 1), (24, 20, 6)]


def _problems(seed=45):
    rng = np.random.default_rng(seed)
    out = []
    for i, (nx, ny, nz) in enumerate(SHAPES):
        d = rng.uniform(2e-9, 4e-9)
        ang = rng.uniform(0, 2 * np.pi)
        b = rng.uniform(0, 50e-3) / MU0
        out.append(dict(cells=(nx, ny, nz), cell_size=(d, d, d), ms=rng.uniform(6e5, 1.2e6),
                        aex=rng.uniform(1e-11, 2e-11), alpha=rng.uniform(0.01, 0.5), gamma=2.211e5,
                        h_ext=(b * np.cos(ang), b * np.sin(ang), 0.0),
                        m0=O.random_unit_vectors(1000 + i, nx * ny * nz)))
    return out


def _oracle(p, dt, n):
    nx, ny, nz = p["cells"]
    prob = O.Problem(nx, ny, nz, *p["cell_size"], ms=p["ms"], aex=p["aex"], alpha=p["alpha"],
                     gamma=p["gamma"], h_ext=p["h_ext"])
    sim = O.Simulation(prob, p["m0"])
    for _ in range(n):
        sim.step(dt)
    return sim.m


@pytest.mark.parametrize("zconv", ["direct", "fft"])
@pytest.mark.parametrize("precision,tol", [(nf.PRECISION_DOUBLE, 1e-10), (nf.PRECISION_SINGLE, 1e-5)])
def test_batch_matches_oracle_per_problem(monkeypatch, precision, tol, zconv):
    if zconv == "fft":
        monkeypatch.setenv("FULLMAG_FDM_BATCH_ZCONV", "fft")
    else:
        monkeypatch.delenv("FULLMAG_FDM_BATCH_ZCONV", raising=False)
    probs = _problems()
    dt, n = 5e-14, 10
    with nf.NativeFdmBatch(probs, precision) as b:
        b.step_n(dt, 4)
        b.step_n(dt, n - 4)   # the graph is replayed; two calls = one trajectory
        tuning = b.tuning()
        assert len(tuning) == 9 and all(g > 0 for g in tuning), tuning
        assert tuning[7] in (128, 256) and tuning[8] in (128, 256), tuning  # x / y tile shape
        for i, p in enumerate(probs):
            err = np.abs(b.copy_m(i) - _oracle(p, dt, n)).max()
            print(i, p["cells"], f"{err:.2e}")
            assert err <= tol, (i, p["cells"], err)


def test_batch_reports_errors():
    bad = _problems()[:2]
    bad[1] = dict(bad[1], ms=0.0)
    with pytest.raises(nf.RunError, match="problem 1: saturation_magnetisation"):
        nf.NativeFdmBatch(bad)
    with nf.NativeFdmBatch(_problems()[:2]) as b:
        with pytest.raises(nf.RunError, match="problem index out of range"):
            b._check(b._lib.fullmag_fdm_batch_copy_m(b._h, 5, np.zeros(3).ctypes.data_as(nf._dp), 3), "copy")


def test_batch_dt_change_matches_oracle():
    probs = _problems()[:3]
    with nf.NativeFdmBatch(probs, nf.PRECISION_DOUBLE) as b:
        b.step_n(5e-14, 3)
        b.step_n(3e-14, 4)
        for i, p in enumerate(probs):
            nx, ny, nz = p["cells"]
            prob = O.Problem(nx, ny, nz, *p["cell_size"], ms=p["ms"], aex=p["aex"], alpha=p["alpha"],
                             gamma=p["gamma"], h_ext=p["h_ext"])
            sim = O.Simulation(prob, p["m0"])
            for dt in [5e-14] * 3 + [3e-14] * 4:
                sim.step(dt)
            assert np.abs(b.copy_m(i) - sim.m).max() <= 1e-10, i
