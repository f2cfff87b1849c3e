#!/usr/bin/env python
"""Benchmark: Heun cell-updates/s of the FP32-mixed path vs the plain FP64 path.

Workload (default, N = 1): 512 x 512 x 8 film of 2 nm cells, Ms = 8e5 A/m,
A = 1.3e-11 J/m, alpha = 0.5, B = (10, 0, 0) mT, seeded random unit m
(seed 43, the planner's generator), Heun dt = 5e-14 s; exchange + demag +
Zeeman.  One "step" is one Heun step of the whole grid (2 097 152 cells).

Reported (one JSON line on rank 0):
  value   FP32-mixed cell-updates/s, whole job, state resident in HBM, timed
          with CUDA events on the library's stream (max over ranks);
  e2e     the same through the C ABI from host buffers: upload of m0 from
          pinned memory, K fullmag_fdm_backend_step calls (stats read back
          every step) and the final copy of m to host, all inside the timed
          region;
  fp64    the plain FP64 path's cell-updates/s and the FP32/FP64 ratio;
  accuracy  max|m_fp32 - m_fp64| from the same m0 at steps 10 ... 2000 (the
          workload's length), each beside FP64's own change from one FP32
          rounding of m0, and the last checkpoint with max|dm| <= 1e-5;
  roofline  the dominant kernel's algorithmic bytes per launch / its mean
          launch time (CUDA events) against the measured HBM copy bandwidth;
  cpu_baseline  the FP64 CPU port of the reference engine (oracle/) timed on
          this host on one Heun step of the same grid.
Multi-GPU: independent replicas (the FFT convolution is global and the
workload does not shard), weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MU0 = 4.0 * np.pi * 1e-7
WORKLOAD = dict(cells=(512, 512, 8), cell_size=(2e-9, 2e-9, 2e-9), ms=8.0e5, aex=1.3e-11,
                alpha=0.5, gamma=2.211e5, b_mT=(10.0, 0.0, 0.0), seed=43, dt=5e-14)
METRIC = "cell-updates/s FP32-mixed vs plain FP64, 1 B200, at max|dm|<=1e-5; HBM GB/s"
ACCURACY_CHECKPOINTS = (10, 50, 100, 200, 500, 1000, 2000)  # up to the workload's 2000 steps
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-ensemble (C4) measurement")
    ap.add_argument("--no-c3", action="store_true", help="skip the large masked DP45 (C3) measurement")
    ap.add_argument("--no-c5", action="store_true", help="skip the adjoint (C5) timing")
    ap.add_argument("--kernels-only", action="store_true",
                    help="FP32-mixed warm-up + K timed steps only (for profiler runs)")
    ap.add_argument("--c3-band", type=int, default=0, metavar="NY",
                    help="profiler run: the C3 geometry cut to 1024 x NY x 16, FP32-mixed DP45, "
                         "K accepted steps after W, per-kernel times of the last")
    return ap.parse_args()


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# --------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples (200 ms) during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        time.sleep(0.25)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------- roofline model
def kernel_bytes(name: str, g: dict, s: int) -> float:
    """Algorithmic bytes of one launch of a library kernel (reads + writes of the
    arrays it must touch once), for the 3-D demag path of grid g."""
    nx, ny, nz = g["cells"]
    n = nx * ny * nz
    nkx, Ly = nx + 1, 2 * ny
    cs = 2 * s
    s1 = 3 * nz * nkx * ny * cs
    s2 = 3 * nz * nkx * Ly * cs
    octant = 6 * (nz + 1) * nkx * (ny + 1) * s
    ztable = 6 * nz * nkx * (ny + 1) * s  # direct z convolution: n(d) for d < nz
    table = {
        "demag_x_fwd": 3 * n * s + s1,
        "demag_y_fwd": s1 + s2,
        "demag_z_conv": 2 * s2 + octant,
        "demag_z_direct": 2 * s2 + ztable,
        "demag_yzy": 2 * s1 + ztable,  # y forward + z + y inverse of a kx plane in shared memory
        "demag_y_inv": s2 + s1,
        "demag_x_inv": s1 + 3 * n * s,
        "stage_combine": 9 * n * s,
        # fused row pass: S1 in and out; RHS: reads m, writes k and the predictor;
        # corrector: reads m_p, m0, k1, writes m (H_d stays in shared memory)
        "row_eval": 2 * s1 + 9 * n * s,
        "row_heun_corr": 2 * s1 + 12 * n * s,
        "row_x_fwd": 3 * n * s + s1,
        "stage_heun_corr": 15 * n * s,   # reads m_p, H_d, m0, k1; writes m
        "stage_eval": 12 * n * s,        # reads m, H_d; writes k and the next predictor
        "reduce_finalize": 0,
    }
    return float(table.get(name, 0))


# --------------------------------------------------------------------- our arm
def run_ours(args):
    import torch

    rank, world, local = env_rank()
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    else:
        torch.cuda.set_device(local)

    from fullmag_b200 import native_fdm as nf

    W = WORKLOAD
    nx, ny, nz = W["cells"]
    n = nx * ny * nz
    K, warm = args.steps, max(3, args.warmup)
    dt = W["dt"]
    m0 = nf.random_unit_vectors(W["seed"], n)
    m0_pinned = torch.from_numpy(m0).pin_memory()
    h = tuple(b * 1e-3 / MU0 for b in W["b_mT"])

    def make(prec):
        plan = nf.FdmPlan(cells=W["cells"], cell_size=W["cell_size"], initial_magnetization=m0,
                          saturation_magnetisation=W["ms"], exchange_stiffness=W["aex"],
                          damping=W["alpha"], gyromagnetic_ratio=W["gamma"], precision=prec,
                          external_field=h, demag_source=nf.DEMAG_NEWELL)
        return nf.NativeFdmBackend(plan)

    def barrier_sync():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.kernels_only:
        be = make(nf.PRECISION_SINGLE)
        be.step_n(dt, warm)
        stream = torch.cuda.ExternalStream(be.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        be.step_n(dt, K)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        if rank == 0:
            print(json.dumps({"mode": "kernels-only", "steps": K, "ms_per_step": ms / K,
                              "value": n * K / (ms * 1e-3)}))
        be.close()
        return

    results = {}
    sampler_out = None
    m_out_pinned = torch.empty(3 * n, dtype=torch.float64).pin_memory()
    for prec, tag in ((nf.PRECISION_DOUBLE, "fp64"), (nf.PRECISION_SINGLE, "fp32")):
        be = make(prec)
        stream = torch.cuda.ExternalStream(be.stream())
        be.step_n(dt, warm)
        # device-resident timing
        barrier_sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(local) if tag == "fp32" else None
        if sampler:
            sampler.__enter__()
        e0.record(stream)
        be.step_n(dt, K)
        e1.record(stream)
        e1.synchronize()
        if sampler:
            sampler.__exit__(None, None, None)
            sampler_out = sampler.summary()
        barrier_sync()
        ms = max_over_ranks(e0.elapsed_time(e1))
        # per-kernel device time (CUDA events around every launch, same stream)
        be.set_profiling(True)
        be.profile_reset()
        be.step_n(dt, K)
        prof = be.profile()
        be.set_profiling(False)
        # end to end through the C ABI from host buffers: upload of m0 from pinned
        # memory, K step calls (statistics read back every step), copy of m into
        # a pinned host array; the three parts are also timed on their own
        barrier_sync()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        be.upload_m(m0_pinned.numpy())
        ev[1].record(stream)
        for _ in range(K):
            be.step(dt)
        ev[2].record(stream)
        be.copy_m(out=m_out_pinned.numpy())
        ev[3].record(stream)
        ev[3].synchronize()
        barrier_sync()
        ms_e2e = max_over_ranks(ev[0].elapsed_time(ev[3]))
        e2e_parts = {"upload_ms": ev[0].elapsed_time(ev[1]), "steps_ms": ev[1].elapsed_time(ev[2]),
                     "download_ms": ev[2].elapsed_time(ev[3])}
        results[tag] = dict(ms=ms, prof=prof, ms_e2e=ms_e2e, e2e_parts=e2e_parts, mem=be.memory_info()[0])
        be.close()
    accuracy = accuracy_table(make, nf, m0, dt)

    s32 = 4
    cells_job = n * K * world
    v32 = cells_job / (results["fp32"]["ms"] * 1e-3)
    v64 = cells_job / (results["fp64"]["ms"] * 1e-3)
    e2e32 = cells_job / (results["fp32"]["ms_e2e"] * 1e-3)

    peak, peak_kind = hbm_peak()
    prof = results["fp32"]["prof"]
    dom = max((k for k in prof if k != "reduce_finalize"), key=lambda k: prof[k][0])
    dom_ms, dom_launch = prof[dom]
    dom_bytes = kernel_bytes(dom, W, s32)
    achieved = dom_bytes / (dom_ms * 1e-3 / dom_launch) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get("fp32", {}).get(dom)
        except Exception:
            traffic = None
    launches = int(sum(c for _, c in prof.values()) // 1)
    step_bytes = sum(kernel_bytes(k, W, s32) * c for k, (_, c) in prof.items()) / K
    kernels = {k: {"ms_per_launch": round(v[0] / v[1], 5), "launches_per_step": v[1] / K,
                   "gbs": round(kernel_bytes(k, W, s32) / (v[0] * 1e-3 / v[1]) / 1e9, 1)}
               for k, v in sorted(prof.items())}
    prof64 = results["fp64"]["prof"]
    kernels64 = {k: {"ms_per_launch": round(v[0] / v[1], 5),
                     "gbs": round(kernel_bytes(k, W, 8) / (v[0] * 1e-3 / v[1]) / 1e9, 1)}
                 for k, v in sorted(prof64.items())}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample()
    batch = None
    if not args.no_batch:
        batch = batch_ensemble_sample()
    c3 = None
    if not args.no_c3:
        c3 = c3_masked_dp45_sample()
    c5 = None
    if not args.no_c5:
        c5 = c5_adjoint_sample()

    if rank == 0:
        bi = 3 * n * 8 / K
        bo = (96 + 3 * n * 8 / K)
        line = {
            "metric": METRIC, "value": v32, "unit": "cell-updates/s", "n_gpus": world,
            "steps": K, "warmup": warm, "ms_per_step": results["fp32"]["ms"] / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32-mixed (f64 Newell setup, renormalisation, energies)",
            "data": "synthetic (seeded random unit m, the reference planner's generator)",
            "config": {"workload": "512x512x8 film, 2 nm cells, Heun dt=5e-14 s, exchange+demag+Zeeman",
                       "cells": n, "padded_fft_xy": [1024, 1024],
                       "y_z_passes": "y forward + direct z sum (nz = 8) + y inverse fused per kx plane, 2-CTA clusters",
                       "parallelism": f"replicas x{world}",
                       "l2": "working set > 126 MB L2 per step (no flush needed)"},
            "fp64": {"value": v64, "ms_per_step": results["fp64"]["ms"] / K,
                     "speedup_fp32_over_fp64": v32 / v64, "kernels": kernels64},
            "accuracy": accuracy,
            "e2e": {"value": e2e32, "unit": "cell-updates/s", "h2d_bytes_per_step": bi,
                    "d2h_bytes_per_step": bo, "steps": K,
                    **{k: round(v, 4) for k, v in results["fp32"]["e2e_parts"].items()},
                    "fixed_ms": round(results["fp32"]["e2e_parts"]["upload_ms"]
                                      + results["fp32"]["e2e_parts"]["download_ms"], 4),
                    "fp64_value": cells_job / (results["fp64"]["ms_e2e"] * 1e-3)},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": f"of {peak_kind}",
                         "algorithmic_bytes_per_launch": dom_bytes, "traffic": traffic,
                         **({"note": "fused kx-plane pass: the x,y spectrum stays in shared memory, so its bytes "
                                     "are S1 in and out plus the z table; the kernel is issue- and latency-bound"}
                            if dom == "demag_yzy" else {})},
            "step_roofline": {"algorithmic_bytes_per_step": step_bytes,
                              "achieved_gbs": step_bytes / (results["fp32"]["ms"] / K * 1e-3) / 1e9,
                              # as built: the bytes the kernels this design runs must move
                              "frac": step_bytes / (results["fp32"]["ms"] / K * 1e-3) / 1e9 / peak,
                              # per cell-update model B_Heun = 2 (78 s + 6 s_k) + 27 s, s = s_k = 4
                              "model_bytes_per_cell_update": 2 * (78 * s32 + 6 * s32) + 27 * s32,
                              "model_achieved_gbs": (2 * (78 * s32 + 6 * s32) + 27 * s32) * (v32 / world) / 1e9,
                              "model_frac": (2 * (78 * s32 + 6 * s32) + 27 * s32) * (v32 / world) / 1e9 / peak},
            "kernels": kernels,
            "gpu_launches": launches,
            "device_bytes": results["fp32"]["mem"],
            "clocks": sampler_out,
            "cpu_baseline": cpu,
            "c4_batch": batch,
            "c3_masked_dp45": c3,
            "c5_adjoint": c5,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def accuracy_table(make, nf, m0, dt):
    """max|m_fp32 - m_fp64| along the workload's 2000 steps from the same m0,
    each beside FP64's own sensitivity: FP64 started from m0 rounded once to
    FP32.  Any FP32-stored state carries at least that rounding, so the floor
    bounds what an FP32-mixed run can reach at that step."""
    a64, a32, f64 = make(nf.PRECISION_DOUBLE), make(nf.PRECISION_SINGLE), make(nf.PRECISION_DOUBLE)
    f64.upload_m(m0.astype(np.float32).astype(np.float64))
    rows, done, last_ok = [], 0, 0
    for k in ACCURACY_CHECKPOINTS:
        for be in (a64, a32, f64):
            be.step_n(dt, k - done)
        done = k
        m64 = a64.copy_m()
        dm = float(np.abs(a32.copy_m() - m64).max())
        fl = float(np.abs(f64.copy_m() - m64).max())
        rows.append({"step": k, "max_dm_fp32_vs_fp64": dm, "fp64_one_fp32_rounding_of_m0": fl})
    for r in rows:  # the gate holds up to the first checkpoint that misses it
        if r["max_dm_fp32_vs_fp64"] > 1e-5:
            break
        last_ok = r["step"]
    for be in (a64, a32, f64):
        be.close()
    return {"rows": rows, "last_checkpoint_with_max_dm_le_1e-5": last_ok,
            "note": "FP32-mixed vs FP64 from the same m0; the floor column is FP64 vs FP64 with m0 "
                    "rounded once to FP32, which no FP32-stored state can avoid"}


# --------------------------------------------------------------------- CPU (oracle) legs
def _oracle_problem(nx, ny, nz):
    from oracle import oracle as O
    W = WORKLOAD
    h = tuple(b * 1e-3 / MU0 for b in W["b_mT"])
    return O, O.Problem(nx, ny, nz, *W["cell_size"], ms=W["ms"], aex=W["aex"], alpha=W["alpha"],
                        gamma=W["gamma"], h_ext=h)


def c3_mask(nx=1024, ny=1024, nz=16, d=2e-9, r_out=1e-6, r_in=150e-9):
    """C3 geometry: a disk of radius 1 um with a centred hole of radius 150 nm
    (300 nm diameter), cell-centre test; Ms = 0 outside."""
    x = (np.arange(nx) + 0.5) * d - nx * d / 2
    y = (np.arange(ny) + 0.5) * d - ny * d / 2
    X, Y = np.meshgrid(x, y)
    r2 = X ** 2 + Y ** 2
    m2 = (r2 <= r_out ** 2) & (r2 > r_in ** 2)
    return np.repeat(m2[None], nz, axis=0).astype(np.uint8).reshape(-1)


def c3_masked_dp45_sample(warm=3, steps=10):
    """C3 on this GPU: 1024 x 1024 x 16 masked film, FP32-mixed DP45 at
    max_error 1e-5 from the planner generator's m0 (seed 44), the suggested dt
    fed back.  `warm` accepted steps untimed, then `steps` accepted steps timed
    with CUDA events on the library's stream, then the same window again with
    per-kernel events.  A window this short starts from the random m0, where
    the accepted dt is smallest, so the time to 5 ns is an upper bound."""
    import torch
    from fullmag_b200 import native_fdm as nf
    nx, ny, nz, d = 1024, 1024, 16, 2e-9
    n = nx * ny * nz
    mask = c3_mask(nx, ny, nz, d)
    active = int(mask.sum())
    m0 = nf.random_unit_vectors(44, n)
    t0 = time.time()
    plan = nf.FdmPlan(cells=(nx, ny, nz), cell_size=(d, d, d), initial_magnetization=m0,
                      saturation_magnetisation=8e5, exchange_stiffness=1.3e-11, damping=0.1,
                      gyromagnetic_ratio=2.211e5, precision=nf.PRECISION_SINGLE, integrator=nf.DP45,
                      external_field=(0.0, 30e-3 / MU0, 0.0), active_mask=mask,
                      adaptive=(1e-5, 1e-18, 1e-10, 0.8), demag_source=nf.DEMAG_NEWELL)
    be = nf.NativeFdmBackend(plan)
    t_create = time.time() - t0
    stream = torch.cuda.ExternalStream(be.stream())
    dt = 1e-13
    for _ in range(warm):
        dt = be.step(dt)["suggested_next_dt"]

    def window(prof):
        nonlocal dt
        if prof:
            be.set_profiling(True)
            be.profile_reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        dts = []
        e0.record(stream)
        for _ in range(steps):
            st = be.step(dt)
            dts.append(st["dt_seconds"])
            dt = st["suggested_next_dt"]
        e1.record(stream)
        e1.synchronize()
        out = (e0.elapsed_time(e1), dts, st)
        if prof:
            out = out + (be.profile(),)
            be.set_profiling(False)
        return out

    ms, dts, st, *_ = window(False)
    _, _, _, prof = window(True)
    be.close()
    s = 4
    D = 78 * s + 6 * s            # bytes per cell of one 3-D demag evaluation (5 passes, octant spectra)
    model = 6 * D + 168 * s       # per cell-update of an accepted DP45 step (FSAL, 6 evaluations)
    peak, peak_kind = hbm_peak()
    v_all = n * steps / (ms * 1e-3)
    attempts = prof.get("stage_dp45_last", (0.0, steps))[1]
    kern = {k: {"ms_per_launch": round(v[0] / v[1], 5), "launches": v[1],
                "share": round(v[0] / sum(x[0] for x in prof.values()), 4)} for k, v in sorted(prof.items())}
    mean_dt = float(np.mean(dts))
    return {"workload": "C3: 1024x1024x16 disk r=1 um with a 150 nm-radius hole (Ms=0 outside), 2 nm cells, "
                        "FP32-mixed DP45 max_error 1e-5, alpha 0.1, B=(0,30,0) mT, seed 44",
            "cells": n, "active_cells": active, "accepted_steps": steps, "warmup_steps": warm,
            "attempts_in_profiled_window": attempts, "rejected_in_profiled_window": attempts - steps,
            "ms_per_accepted_step": ms / steps, "value": v_all, "unit": "cell-updates/s",
            "active_cell_updates_per_s": active * steps / (ms * 1e-3),
            "mean_dt_s": mean_dt, "sim_time_in_window_s": float(np.sum(dts)),
            "extrapolated_s_to_5ns_at_this_dt": 5e-9 / mean_dt * ms * 1e-3 / steps,
            "model_bytes_per_cell_update": model,
            "model_frac": model * v_all / 1e9 / peak, "peak_gbs": peak, "peak_kind": f"of {peak_kind}",
            "kernels": kern, "create_s": t_create,
            "note": "the window starts from random m0, where dt is smallest; the 5 ns figure is an upper bound"}


def c5_adjoint_sample(steps=2000):
    """C5 on this GPU: 256 x 256 x 1 film of 4 x 4 x 3 nm cells, per-cell Ms
    ~ U[6e5, 1e6] (seed 46), A 1.3e-11, alpha 0.05, B(t) = (20 sin(2 pi 5 GHz t),
    0, 5) mT, Heun dt 1e-13 x 2000, loss = sum of m_x over the central 64 x 64.
    Per precision, CUDA events on the library's stream around: the 2000 forward
    steps alone; the forward with sqrt(N) device checkpoints; the backward pass
    (segment replays from the checkpoints, then the adjoint steps)."""
    import torch
    from fullmag_b200 import native_fdm as nf
    nx = ny = 256
    rng = np.random.default_rng(46)
    ms_map = rng.uniform(6e5, 1e6, nx * ny)
    m0 = np.tile([0.0, 1.0, 0.0], nx * ny)
    sel = np.zeros((ny, nx), bool)
    sel[96:160, 96:160] = True
    g = np.zeros((nx * ny, 3))
    g[sel.reshape(-1), 0] = 1.0
    out = {"workload": "C5: 256x256x1, 4x4x3 nm, Ms map U[6e5,1e6], B(t)=(20 sin(2pi 5GHz t),0,5) mT, "
                       "Heun dt 1e-13 x 2000, loss = sum m_x over the central 64x64",
           "steps": steps, "checkpoints": int(np.ceil(np.sqrt(steps)))}
    for prec, tag in ((nf.PRECISION_DOUBLE, "fp64"), (nf.PRECISION_SINGLE, "fp32")):
        plan = nf.FdmPlan(cells=(nx, ny, 1), cell_size=(4e-9, 4e-9, 3e-9), initial_magnetization=m0,
                          exchange_stiffness=1.3e-11, damping=0.05, gyromagnetic_ratio=2.211e5,
                          precision=prec, external_field=(0.0, 0.0, 5e-3 / MU0), ms_map=ms_map,
                          ac_field=(20e-3 / MU0, 0.0, 0.0), ac_frequency_hz=5e9, demag_source=nf.DEMAG_NEWELL)
        be = nf.NativeFdmBackend(plan)
        stream = torch.cuda.ExternalStream(be.stream())
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        be.step_n(1e-13, 5)  # warm-up
        be.upload_m(m0)
        ev[0].record(stream)
        be.step_n(1e-13, steps)
        ev[1].record(stream)
        be.upload_m(m0)
        ev[2].record(stream)
        be.adjoint_forward(1e-13, steps)
        ev[3].record(stream)
        grads = be.adjoint_backward(g.reshape(-1))
        ev[4].record(stream)
        ev[4].synchronize()
        fwd, fwd_ck, bwd = ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3]), ev[3].elapsed_time(ev[4])
        out[tag] = {"forward_ms": fwd, "forward_with_checkpoints_ms": fwd_ck, "backward_ms": bwd,
                    "backward_over_forward": bwd / fwd, "checkpoint_overhead": fwd_ck / fwd - 1.0,
                    "dl_dms_abs_max": float(np.abs(grads["dl_dms"]).max()),
                    "dl_dh_ext": [float(v) for v in grads["dl_dh_ext"]]}
        be.close()
    return out


def c4_problems(count=256, seed=45):
    """Config C4: 256 problems, nx ~ U{32..256}, ny ~ U{32..128}, nz ~ U{1..4},
    isotropic cells ~ U[2, 4] nm, Ms ~ U[6e5, 1.2e6] A/m, A ~ U[1e-11, 2e-11] J/m,
    alpha ~ U[0.01, 0.5], |B| ~ U[0, 50] mT at a uniform in-plane angle, seeded
    random m0 per problem."""
    import numpy as np
    from fullmag_b200 import native_fdm as nf
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        nx, ny, nz = int(rng.integers(32, 257)), int(rng.integers(32, 129)), int(rng.integers(1, 5))
        d = rng.uniform(2e-9, 4e-9)
        ang, b = rng.uniform(0, 2 * np.pi), rng.uniform(0, 50e-3) / MU0
        out.append(dict(cells=(nx, ny, nz), cell_size=(d, d, d), ms=rng.uniform(6e5, 1.2e6),
                        aex=rng.uniform(1e-11, 2e-11), alpha=rng.uniform(0.01, 0.5),
                        h_ext=(b * np.cos(ang), b * np.sin(ang), 0.0),
                        m0=nf.random_unit_vectors(seed * 1000 + i, nx * ny * nz)))
    return out


def _pow2_at_least(v):
    p = 1
    while p < v:
        p *= 2
    return p


def _batch_length(v, dbl=False):
    """The batch's padded in-plane length (batch.cu batch_length): at least 16,
    the smallest power of two >= v, or in FP32 3 * 2^k in 96..768 when shorter."""
    L = max(16, _pow2_at_least(v))
    if not dbl:
        for c in (96, 192, 384, 768):
            if v <= c < L:
                L = c
    return L


def batch_kind_bytes(probs, s=4, zdirect=True):
    """Algorithmic bytes per Heun step of each batched kernel kind (x fwd, y fwd,
    z, y inv, x inv, stage; both evaluations of a step), summed over the
    problems with the batch's padding (in-plane lengths as batch_length, z to a
    power of two >= 2 nz).  The z kind reads the direct table (nz planes per
    component) or, with the z FFT, the octant (Lz / 2 + 1 planes)."""
    tot = [0.0] * 6
    cs = 2 * s
    for p in probs:
        nx, ny, nz = p["cells"]
        n = nx * ny * nz
        Lx, Ly, Lz = _batch_length(2 * nx, s == 8), _batch_length(2 * ny, s == 8), _pow2_at_least(2 * nz)
        nkx = Lx // 2 + 1
        s1 = 3 * nz * nkx * ny * cs
        s2 = 3 * nz * nkx * Ly * cs
        table = 6 * (nz if zdirect else Lz // 2 + 1) * nkx * (Ly // 2 + 1) * s
        per_eval = [3 * n * s + s1, s1 + s2, 2 * s2 + table, s2 + s1, s1 + 3 * n * s]
        for k in range(5):
            tot[k] += 2 * per_eval[k]
        tot[5] += (12 + 15) * n * s  # RHS (+ predictor) and corrector
    return tot


def batch_ensemble_sample(steps=1000):
    """C4 on this GPU: FP32-mixed Heun dt 5e-14 through fullmag_fdm_batch_*
    (one persistent launch per stage, one CUDA graph per step); 10 warm-up steps
    (autotuner + graph capture), then `steps` steps timed with CUDA events on the
    batch's stream, then one step with its launches timed by kind."""
    import torch
    from fullmag_b200 import native_fdm as nf
    probs = c4_problems()
    cells = int(sum(p["cells"][0] * p["cells"][1] * p["cells"][2] for p in probs))
    t0 = time.time()
    b = nf.NativeFdmBatch(probs, nf.PRECISION_SINGLE)
    t_create = time.time() - t0
    b.step_n(5e-14, 10)
    stream = torch.cuda.ExternalStream(b.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step_n(5e-14, steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    kinds = b.profile_step(5e-14)
    tuning = b.tuning()
    b.close()
    names = ["x_fwd", "y_fwd", "z_conv", "y_inv", "x_inv", "stage"]
    kb = batch_kind_bytes(probs, zdirect=os.environ.get("FULLMAG_FDM_BATCH_ZCONV") != "fft")
    peak, peak_kind = hbm_peak()
    per_kind = {nm: {"ms_per_step": round(kinds[i], 5), "gbs": round(kb[i] / (kinds[i] * 1e-3) / 1e9, 1)}
                for i, nm in enumerate(names)}
    dom = max(range(6), key=lambda i: kinds[i])
    step_bytes = sum(kb)
    return {"workload": "C4: 256 problems, grids U{32..256} x U{32..128} x U{1..4}, FP32-mixed Heun dt 5e-14",
            "problems": len(probs), "cells": cells, "steps": steps, "value": cells * steps / (ms * 1e-3),
            "unit": "cell-updates/s", "ms_per_step": ms / steps, "create_s": t_create,
            "kernels": per_kind,
            "roofline": {"kernel": names[dom], "achieved": kb[dom] / (kinds[dom] * 1e-3) / 1e9, "peak": peak,
                         "frac": kb[dom] / (kinds[dom] * 1e-3) / 1e9 / peak, "unit": "GB/s",
                         "peak_kind": f"of {peak_kind}"},
            "step_bytes": step_bytes, "step_frac": step_bytes / (ms / steps * 1e-3) / 1e9 / peak,
            "autotuned_grid": tuning,
            "timing": "CUDA events on the batch stream around step_n (graph replays); per-kind split from "
                      "one step with the launches issued one by one"}


def cpu_baseline_sample():
    """One Heun step of the full grid on the FP64 CPU port (about 10-30 s)."""
    O, p = _oracle_problem(*WORKLOAD["cells"])
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    nx, ny, nz = WORKLOAD["cells"]
    sim = O.Simulation(p, O.random_unit_vectors(WORKLOAD["seed"], nx * ny * nz))
    t0 = time.perf_counter()
    sim.step(WORKLOAD["dt"])
    el = time.perf_counter() - t0
    return {"value": nx * ny * nz / el, "unit": "cell-updates/s", "cores": threads, "kind": "port",
            "sample": f"1 Heun step of the full {nx}x{ny}x{nz} grid, FP64, OpenMP pointwise loops, "
                      f"serial FFT lines as in the reference ({el:.1f} s)"}


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return
    O = None
    threads = os.cpu_count() or 1
    # bounded sample per step: the largest film of the workload's shape whose
    # W + K steps fit in about three minutes of this host's CPU time
    nx, ny, nz = WORKLOAD["cells"]
    O, p = _oracle_problem(64, 64, nz)
    O.set_threads(threads)
    sim = O.Simulation(p, O.random_unit_vectors(WORKLOAD["seed"], 64 * 64 * nz))
    t0 = time.perf_counter()
    sim.step(WORKLOAD["dt"])
    per_cell = (time.perf_counter() - t0) / (64 * 64 * nz)
    budget = 180.0 / (args.steps + max(3, args.warmup))
    side = 64
    while side * 2 <= nx and per_cell * 1.3 * (2 * side) ** 2 * nz <= budget:
        side *= 2
    O, p = _oracle_problem(side, side, nz)
    sim = O.Simulation(p, O.random_unit_vectors(WORKLOAD["seed"], side * side * nz))
    for _ in range(max(3, args.warmup)):
        sim.step(WORKLOAD["dt"])
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.step(WORKLOAD["dt"])
    el = time.perf_counter() - t0
    v = side * side * nz * args.steps / el
    sample = (f"{side}x{side}x{nz} film with the workload's physics (the full 512x512x8 grid "
              f"takes ~{per_cell * 1.3 * nx * ny * nz:.0f} s per step here); FP64 CPU port of the "
              f"reference engine, OpenMP pointwise loops, serial FFT lines")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded random unit m)",
            "config": {"workload": "512x512x8 film, 2 nm cells, Heun dt=5e-14 s, exchange+demag+Zeeman",
                       "sample_grid": [side, side, nz], "parallelism": "host CPU"},
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def c3_band_run(ny, steps, warm):
    """The C3 geometry cut to a 1024 x ny x 16 band (ny <= 1024; the disk
    centred in the band), FP32-mixed DP45 as in c3_masked_dp45_sample: `warm`
    accepted steps, then `steps` more with per-kernel CUDA events; prints one
    JSON line.  A case for profiler captures that holds a few GB at most."""
    import torch  # noqa: F401  (CUDA context through the library)
    from fullmag_b200 import native_fdm as nf
    nx, nz, d = 1024, 16, 2e-9
    n = nx * ny * nz
    mask = c3_mask(nx, ny, nz, d)
    plan = nf.FdmPlan(cells=(nx, ny, nz), cell_size=(d, d, d), initial_magnetization=nf.random_unit_vectors(44, n),
                      saturation_magnetisation=8e5, exchange_stiffness=1.3e-11, damping=0.1,
                      gyromagnetic_ratio=2.211e5, precision=nf.PRECISION_SINGLE, integrator=nf.DP45,
                      external_field=(0.0, 30e-3 / MU0, 0.0), active_mask=mask,
                      adaptive=(1e-5, 1e-18, 1e-10, 0.8), demag_source=nf.DEMAG_NEWELL)
    be = nf.NativeFdmBackend(plan)
    dt = 1e-13
    for _ in range(warm):
        dt = be.step(dt)["suggested_next_dt"]
    be.set_profiling(True)
    for _ in range(steps):
        dt = be.step(dt)["suggested_next_dt"]
    prof = be.profile()
    be.close()
    print(json.dumps({"mode": "c3-band", "cells": [nx, ny, nz], "steps": steps,
                      "kernels_ms_per_launch": {k: v[0] / v[1] for k, v in sorted(prof.items())}}))


def main():
    args = parse()
    if args.c3_band:
        c3_band_run(args.c3_band, args.steps, args.warmup)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
