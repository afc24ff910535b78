#!/usr/bin/env python
"""bench.py -- homogenized C^H (+ dC^H/drho) per second at 128^3 on B200.

One step = one periodic six-load-case homogenization of a 128^3 cell
(6.29 M DOF, all six right-hand sides) in mixed precision (FP64 CG and FP64
operator, FP32 multigrid V-cycle preconditioner: stencil sweeps, residuals and
transfers in FP32; FP64 inner products, FP64 coarse solve; FP64 relative
residual 1e-10) plus the adjoint gradient dL/drho of L = ||C^H - C_t||_F^2 --
the engine's C ABI (femh_homogenize + femh_homogenize_grad), called from this
process.  The FP32-inner-solve defect-correction variant is reported beside it.

Lines printed (rank 0):
  default            {"metric": ..., "value": tensors(+grad)/s, ...}
  --impl reference   the reference path's CPU implementation (the FP64 oracle
                     port: Jacobi-PCG, OpenMP) on the host cores, same metric.

Workload: seeded synthetic 128^3 cell (periodic white noise, Gaussian filter
sigma = 4 voxels, sigmoid slope 4, mapped to [1e-3, 1]); the target C_t is the
C^H of an independent seeded cell.  Inputs (and every solver vector, >= 150 MB
each) are larger than the 126 MB L2.
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

METRIC = "Homogenized C(+dC/drho)/s at 128^3, <=1e-6 rel err: mixed vs plain FP64 on B200"
UNIT = "tensors+grad/s"
N = 128


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="femh", choices=["femh", "reference"])
    ap.add_argument("--n", type=int, default=N)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-autotune", action="store_true",
                    help="heuristic tile shapes (the first stencil launches are then the solve's own)")
    ap.add_argument("--quick", action="store_true",
                    help="timed device steps only (no e2e / FP64 / roofline / CPU legs): the profiling command")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks --
class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ----------------------------------------------------------- CPU baseline --
def cpu_baseline(rho, Ct, jacobi_iters: int, sample_iters: int = 2):
    """The oracle port (FP64 Jacobi-PCG, matrix-free, OpenMP) on this host:
    `sample_iters` PCG iterations of all six load cases at full size plus one
    energy and one gradient pass, extrapolated to `jacobi_iters` iterations
    (the count the same algorithm needs on this field)."""
    from oracle import oracle as O
    mat = O.material()
    n = rho.shape[0]
    h = 1.0 / n
    t_iter = O.time_pcg(rho, sample_iters, mat, h)
    chi = np.zeros((6,) + rho.shape + (3,))
    t1 = time.perf_counter()
    C = O.energy(rho, chi, h, mat)
    O.grad(rho, chi, 2 * (C - Ct), h, mat)
    t_post = time.perf_counter() - t1
    total = t_iter * jacobi_iters + t_post
    return {
        "value": 1.0 / total, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
        "sample": (f"{sample_iters} Jacobi-PCG iterations x 6 load cases at {n}^3 FP64 "
                   f"({t_iter:.3f} s/iteration) + 1 energy + 1 gradient pass ({t_post:.2f} s), "
                   f"extrapolated to the {jacobi_iters} iterations this algorithm needs on the field"),
        "seconds_per_tensor": total,
    }


def jacobi_iteration_count(rho) -> int:
    """Iterations of FP64 Jacobi-PCG to 1e-10 on this field (max over load
    cases), counted by the GPU engine running the same algorithm in FP64."""
    import fem_b200 as F
    e = F.Engine(F.Config(solver=F.JACOBI_PCG, precision=F.FP64, max_iter=200000))
    C, info = e.homogenize(rho, allow_unconverged=True)
    e.close()
    return int(max(info["iterations"]))


# ----------------------------------------------------------------- main ---
def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    from fem_b200 import fields

    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    from fem_b200 import build
    build.build()
    import fem_b200 as F
    from fem_b200.dist import max_over_ranks

    n = args.n
    rho_h = fields.smooth_cell(n, 4.0, seed=2 + rank)
    Ct = F.Engine(F.Config(device=local)).homogenize(fields.smooth_cell(n, 4.0, seed=5))[0]

    stream = torch.cuda.current_stream()
    cfg = F.Config(device=local, precision=F.MIXED_PC, solver=F.GMG_PCG, autotune=0 if args.no_autotune else 1)
    eng = F.Engine(cfg)
    eng.set_stream(stream.cuda_stream)
    rho_d = torch.from_numpy(rho_h).cuda()
    grad_d = torch.empty_like(rho_d)

    def step_dev():
        C, info = eng.homogenize(rho_d)
        eng.grad(2 * (C - Ct), out=grad_d)
        return C, info

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps, tag="timed"):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push(tag)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), device="cuda")
        barrier()
        return ms

    for _ in range(args.warmup if args.quick else max(3, args.warmup)):
        C_mixed, info = step_dev()
    launches0 = eng.kernel_launches
    with ClockSampler(local) as clk:
        ms = timed(step_dev, args.steps)
    gpu_launches = eng.kernel_launches - launches0
    ms_step = ms / args.steps
    value = world * args.steps / (ms / 1e3)
    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "ms_per_step": ms_step,
                              "quick": True, "gpu_launches": gpu_launches}), flush=True)
        return

    # end-to-end: host buffers through the C ABI (H2D of rho, D2H of C and dL/drho)
    import ctypes
    pin_rho = torch.from_numpy(rho_h).pin_memory()
    pin_grad = torch.empty_like(pin_rho).pin_memory()
    rho_pin_np = pin_rho.numpy()
    grad_pin_np = pin_grad.numpy()

    def step_e2e():
        C, info = eng.homogenize(rho_pin_np)
        eng.grad(2 * (C - Ct), out=grad_pin_np)
    for _ in range(2):
        step_e2e()
    e2e_ms = timed(step_e2e, args.steps, "e2e") / args.steps
    e2e_val = world / (e2e_ms / 1e3)
    h2d = rho_h.nbytes
    d2h = 36 * 8 + rho_h.nbytes

    # plain FP64 GPU PCG, same step (the comparison the metric names)
    eng64 = F.Engine(F.Config(device=local, precision=F.FP64, solver=F.GMG_PCG))
    eng64.set_stream(stream.cuda_stream)
    grad64 = torch.empty_like(rho_d)

    def step64():
        C, info = eng64.homogenize(rho_d)
        eng64.grad(2 * (C - Ct), out=grad64)
        return C, info
    C64, info64 = step64()
    k64 = max(1, min(3, args.steps))
    ms64 = timed(step64, k64, "fp64") / k64
    C64, info64 = step64()
    rel_err = float(np.abs(C_mixed - C64).max() / np.abs(C64).max())

    # defect-correction variant (FP32 inner PCG solves inside FP64 refinement)
    engdc = F.Engine(F.Config(device=local, precision=F.MIXED, solver=F.GMG_PCG, inner_tol=1e-3))
    engdc.set_stream(stream.cuda_stream)
    graddc = torch.empty_like(rho_d)

    def stepdc():
        C, info = engdc.homogenize(rho_d)
        engdc.grad(2 * (C - Ct), out=graddc)
        return C, info
    Cdc, infodc = stepdc()
    msdc = timed(stepdc, k64, "dc") / k64
    engdc.close()

    # roofline of the dominant kernel: one profiled step (CUDA events per launch)
    eng.profile(True)
    step_dev()
    stats = eng.profile_read()
    eng.profile(False)
    tot_ms = sum(s["total_ms"] for s in stats)
    top = max(stats, key=lambda s: s["total_ms"])
    peak, peak_kind = measured_peaks()
    per_launch_ms = top["total_ms"] / top["launches"]
    per_launch_bytes = top["bytes"] / top["launches"]
    achieved = per_launch_bytes / (per_launch_ms / 1e3) / 1e9 if per_launch_bytes > 0 else 0.0
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        traffic = json.load(open(tfile)).get(top["name"].split("_L")[0])

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 preconditioner / f64 CG",
        "data": "synthetic (seeded filtered-noise densities)",
        "config": {"workload": f"{n}^3 periodic cell, smooth rho in [1e-3,1] (sigma 4), 6 load cases, "
                               f"FP64 CG + FP32 GMG V-cycle to 1e-10 + adjoint dL/drho",
                   "grid": n, "dof": 3 * n ** 3, "rhs": 6, "solver": "GMG-PCG (Jacobi 3+3 with Chebyshev-root "
                   "weights, rediscretised coarse levels, FP64 dense coarse solve)",
                   "l2": "inputs and vectors larger than L2 (no flush needed)",
                   "parallelism": f"replicas x{world} (independent cells, one per GPU)"},
        "clocks": clk.summary(),
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": gpu_launches,
        "solve": {"outer_iterations": info["outer_iterations"], "inner_iterations": info["iterations"],
                  "rel_residual": max(info["rel_residual"]),
                  # 3 n^3 DOF times the six load cases' CG iterations, per second of
                  # the step (rank 0's counts times the ranks)
                  "dof_iterations_per_s": world * 3 * n ** 3 * sum(info["iterations"]) / (ms_step / 1e3)},
        "mixed_defect_correction": {"ms_per_step": msdc, "value": world / (msdc / 1e3),
                                    "outer_iterations": infodc["outer_iterations"],
                                    "inner_iterations": infodc["iterations"],
                                    "C_rel_err_vs_fp64": float(np.abs(Cdc - C64).max() / np.abs(C64).max())},
        "fp64_plain": {"ms_per_step": ms64, "value": world / (ms64 / 1e3),
                       "iterations": info64["iterations"], "mixed_speedup": ms64 / ms_step,
                       "dof_iterations_per_s": world * 3 * n ** 3 * sum(info64["iterations"]) / (ms64 / 1e3),
                       "C_rel_err_mixed_vs_fp64": rel_err},
        "roofline": {"bound": "hbm", "kernel": top["name"], "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind, "share_of_step": top["total_ms"] / tot_ms,
                     "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms},
        "kernels": sorted(({"name": s["name"], "launches": s["launches"], "ms": round(s["total_ms"], 4),
                            "share": round(s["total_ms"] / tot_ms, 4)} for s in stats),
                          key=lambda d: -d["ms"])[:12],
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        it = jacobi_iteration_count(rho_h)
        out["cpu_baseline"] = cpu_baseline(rho_h, Ct, it)
    if rank == 0:
        print(json.dumps(out), flush=True)
    eng.close()
    eng64.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args, world, rank):
    """The reference path's CPU implementation (the oracle port) on the host
    cores; rank 0 alone runs and prints, other ranks exit without work."""
    if rank != 0:
        return
    from fem_b200 import fields
    n = args.n
    rho = fields.smooth_cell(n, 4.0, seed=2)
    from oracle import oracle as O
    O.build()
    Ct = O.c_iso(0.05, 0.3)
    try:
        it = jacobi_iteration_count(rho)
        src = "counted by the GPU engine running the same FP64 Jacobi-PCG"
    except Exception:
        it = 4 * max(O.homogenize(fields.smooth_cell(32, 1.0, seed=2))[2])
        src = "estimated as 4x the 32^3 count (no GPU)"
    vals = []
    for s in range(args.warmup + args.steps):
        cb = cpu_baseline(rho, Ct, it, sample_iters=1)
        if s >= args.warmup:
            vals.append(cb["seconds_per_tensor"])
    sec = statistics.median(vals)
    cb["sample"] += f"; iteration count {src}"
    out = {
        "metric": METRIC, "value": 1.0 / sec, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded filtered-noise densities)",
        "impl": "reference",
        "config": {"workload": f"{n}^3 periodic cell, smooth rho in [1e-3,1] (sigma 4), 6 load cases, "
                               f"FP64 Jacobi-PCG to 1e-10 + dL/drho (CPU oracle port)", "grid": n},
        "cpu_baseline": {"value": 1.0 / sec, "unit": UNIT, "cores": cb["cores"], "kind": "port",
                         "sample": cb["sample"]},
        "e2e": {"value": 1.0 / sec, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
