"""The batched ensemble on the benchmark's own draw: the 256 problems of the C4
configuration (bench.c4_problems, seed 45: grids U{32..256} x U{32..128} x
U{1..4}, cells U[2, 4] nm, uneven materials and fields), stepped together in
FP32-mixed Heun at dt = 5e-14 s.  After 5 steps the 4 largest problems and 4
drawn at random are compared with the FP64 oracle run alone on each, at the
FP32-mixed bound of the other parity tests (max|dm| <= 1e-5).  (The oracle's
serial FFT lines make each of the largest problems' steps take seconds.)"""
import numpy as np
import pytest

from fullmag_b200 import native_fdm as nf
from oracle import oracle as O

import bench

pytestmark = pytest.mark.gpu


def _oracle(p, dt, n):
    nx, ny, nz = p["cells"]
    prob = O.Problem(nx, ny, nz, *p["cell_size"], ms=p["ms"], aex=p["aex"], alpha=p["alpha"],
                     gamma=p.get("gamma", 2.211e5), h_ext=p["h_ext"])
    sim = O.Simulation(prob, p["m0"])
    for _ in range(n):
        sim.step(dt)
    return sim.m


def test_c4_draw_largest_and_random_problems_match_oracle():
    import os
    O.set_threads(os.cpu_count() or 1)
    probs = bench.c4_problems()
    assert len(probs) == 256
    sizes = np.array([p["cells"][0] * p["cells"][1] * p["cells"][2] for p in probs])
    largest = list(np.argsort(sizes)[-4:])
    rng = np.random.default_rng(2024)
    rest = [i for i in range(256) if i not in largest]
    picked = largest + list(rng.choice(rest, 4, replace=False))
    dt, n = 5e-14, 5
    with nf.NativeFdmBatch(probs, nf.PRECISION_SINGLE) as b:
        b.step_n(dt, n)
        for i in picked:
            err = float(np.abs(b.copy_m(int(i)) - _oracle(probs[i], dt, n)).max())
            print(int(i), probs[i]["cells"], f"{err:.2e}")
            assert err <= 1e-5, (int(i), probs[i]["cells"], err)
