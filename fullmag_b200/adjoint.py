"""torch.autograd.Function over the library's Heun trajectory and its adjoint.

    m_final = HeunTrajectory.apply(m0, ms_map, h_ext, h_ac, problem, dt, n_steps, checkpoint_every)

`m0` (N, 3), `ms_map` (N,), `h_ext` (3,) and `h_ac` (3,) are float64 tensors
(A/m for the fields; H(t) = h_ext + h_ac sin(2 pi f t)); `problem` is a dict of
the remaining FdmPlan fields (cells, cell_size, exchange_stiffness, damping,
gyromagnetic_ratio, precision, ac_frequency_hz, active_mask, ...).  The
forward pass creates a backend, takes n_steps Heun steps through
fullmag_fdm_adjoint_forward (device checkpoints every checkpoint_every steps,
0 = ceil(sqrt(n_steps))) and returns m_final (N, 3); the backward pass runs
fullmag_fdm_adjoint_backward with the incoming dL/dm_final and returns
dL/dm0, dL/dMs, dL/dh_ext and dL/dh_ac.  All arithmetic happens in the CUDA
library; torch only carries the tensors.
"""
from __future__ import annotations

import numpy as np
import torch

from . import native_fdm as nf


class HeunTrajectory(torch.autograd.Function):
    @staticmethod
    def forward(ctx, m0, ms_map, h_ext, h_ac, problem: dict, dt: float, n_steps: int,
                checkpoint_every: int = 0):
        kw = dict(problem)
        kw.setdefault("demag_source", nf.DEMAG_NEWELL)
        plan = nf.FdmPlan(initial_magnetization=m0.detach().cpu().double().numpy().reshape(-1),
                          ms_map=ms_map.detach().cpu().double().numpy(),
                          external_field=tuple(float(v) for v in h_ext.detach().cpu()),
                          ac_field=tuple(float(v) for v in h_ac.detach().cpu()), **kw)
        be = nf.NativeFdmBackend(plan)
        be.adjoint_forward(dt, int(n_steps), int(checkpoint_every))
        ctx.backend = be
        ctx.n = plan.cell_count
        return torch.from_numpy(be.copy_m().reshape(-1, 3)).to(m0.device)

    @staticmethod
    def backward(ctx, grad_m):
        be = ctx.backend
        g = be.adjoint_backward(grad_m.detach().cpu().double().numpy().reshape(-1))
        be.close()
        ctx.backend = None
        dev = grad_m.device
        return (torch.from_numpy(g["dl_dm0"].reshape(-1, 3)).to(dev), torch.from_numpy(g["dl_dms"]).to(dev),
                torch.from_numpy(g["dl_dh_ext"]).to(dev), torch.from_numpy(g["dl_dh_ac"]).to(dev),
                None, None, None, None)
