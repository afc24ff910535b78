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
                     port: the same multigrid PCG, OpenMP) on the host cores,
                     same metric and workload, converged solves measured.

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
    ap.add_argument("--no-batch", action="store_true", help="skip the uneven 4096-cell batch leg")
    ap.add_argument("--batch-cells", type=int, default=4096, help="cells of the uneven batch leg")
    ap.add_argument("--no-autotune", action="store_true",
                    help="heuristic tile shapes (the first stencil launches are then the solve's own)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="plain launches instead of the CUDA-graph loop (ncu cannot profile kernels inside a "
                         "graph with conditional nodes): the launch-list command")
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


# The headers a kernel family is compiled from: the stencil kernels include
# only these two; every other kernel is hashed over all the headers.
KERNEL_HEADERS = {"stencil_": ("femh_common.cuh", "stencil.cuh")}


def engine_source_sha(kernel: str | None = None) -> str:
    """Hash of the device code `kernel` is compiled from (the kernel headers of
    fem_b200/csrc it includes; all of them when kernel is None): ties a
    DRAM-traffic capture to the code it measured."""
    import hashlib
    h = hashlib.sha256()
    base = os.path.join(ROOT, "fem_b200", "csrc")
    files = sorted(f for f in os.listdir(base) if f.endswith(".cuh"))
    for prefix, hdrs in KERNEL_HEADERS.items():
        if kernel is not None and kernel.startswith(prefix):
            files = sorted(hdrs)
    for f in files:
        h.update(open(os.path.join(base, f), "rb").read())
    return h.hexdigest()[:16]


def kernel_traffic(kernel: str):
    """DRAM bytes (read + write) per launch of the dominant kernel from the ncu
    capture recorded in profiles/traffic.json -- only when that capture was
    taken of these very sources; else None."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None, "no ncu capture recorded"
    d = json.load(open(path))
    if d.get("source_sha") != engine_source_sha(kernel):
        return None, "recorded ncu capture is of other engine sources"
    v = d.get("kernels", {}).get(kernel)
    return (v, d.get("how", "")) if v is not None else (None, f"no ncu capture of {kernel}")


# ----------------------------------------------------------- CPU baseline --
SOLVER = ("GMG-PCG, block CG over the six load cases (6x6 steps, FP64 search directions): node-block (3x3) "
          "Jacobi 3+3 sweeps with Chebyshev-root weights, rediscretised coarse levels down to <= 64 nodes, FP64 "
          "dense coarse solve")


def workload_config(n: int, world: int) -> dict:
    """The workload both arms run (the reference arm on the host cores)."""
    return {"workload": f"{n}^3 periodic cell, smooth rho in [1e-3,1] (sigma 4, seed 2), 6 load cases solved to an "
                        f"FP64 relative residual of 1e-10, C^H, then dL/drho of L = ||C^H - C_t||_F^2",
            "grid": n, "dof": 3 * n ** 3, "rhs": 6, "solver": SOLVER,
            "l2": "inputs and vectors larger than L2 (no flush needed)",
            "parallelism": f"replicas x{world} (independent cells, one per GPU)"}


def cpu_baseline(rho, Ct):
    """The oracle port on this host, measured: one converged FP64 multigrid-PCG
    solve of the six load cases (oracle/femh_oracle_mg.c -- the same V-cycle
    as the GPU path), the energy reduction to C^H and the adjoint gradient."""
    from oracle import oracle as O
    n = rho.shape[0]
    t0 = time.perf_counter()
    C, chi, it, rel, st = O.mg_homogenize(rho, tol=1e-10, block=True)
    t1 = time.perf_counter()
    O.grad(rho, chi, 2 * (C - Ct))
    t2 = time.perf_counter()
    total = t2 - t0
    return {
        "value": 1.0 / total, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
        "sample": (f"measured: one converged FP64 multigrid-PCG solve at {n}^3 (6 load cases, "
                   f"{max(it)} iterations, relative residual {max(rel):.1e}, {t1 - t0:.1f} s incl. C^H) "
                   f"+ one adjoint gradient pass ({t2 - t1:.1f} s); oracle/femh_oracle_mg.c, OpenMP"),
        "seconds_per_tensor": total, "iterations": it, "status": st,
    }


# ----------------------------------------------------- uneven batch leg --
# Share of the device's free memory one batched call may plan for (the
# engine's estimate covers its arrays; the rest is the CUDA context, the
# gradient output and unit tables, ~2 GB at 4096 cells).
FIT = 0.95


def batched_uneven(F, local: int, ncell: int, world: int = 1, rank: int = 0, fp64_sample: int = 128) -> dict:
    """The seeded uneven set (n in {16,24,32,48,64}, binary voxels, volume
    fraction U[0.2,0.6]) solved in mixed precision in as few batched calls as
    fit the device (one for the 4096 cells on one B200), with dC^H/drho
    contracted against a fixed weight tensor per cell (the adjoint pass),
    against solving cells one at a time with the plain FP64 path (set-up
    included, timed on the first `fp64_sample` cells, rank 0).  With several
    ranks the cells are sharded by voxels (fem_b200.dist.shard, no data-path
    collective) and the time is the max over ranks.  Wall time around the calls
    (each call ends with its results on the host)."""
    from fem_b200 import fields
    from fem_b200.dist import max_over_ranks, shard
    cells = fields.uneven_batch(4096, seed=7, count=ncell)
    mine = shard([float(c.size) for c in cells], world)[rank]
    my_cells = [cells[i] for i in mine]
    W = np.tile(np.diag([1.0, 1.0, 1.0, 0.5, 0.5, 0.5]), (len(my_cells), 1, 1))
    # the defaults (block PCG over the load cases, FP64 search directions;
    # node-block smoothing) where the set fits one call with them; otherwise
    # the first of point smoothing / one-case PCG (FP32 directions) that fits
    choices = [(1, 1), (1, 0), (0, 1), (0, 0)]   # (block_cg, block_jacobi)
    need0 = None
    for bc, bj in choices:
        e = F.Engine(F.Config(device=local, precision=F.MIXED_PC, block_cg=bc, block_jacobi=bj))
        need, avail = e.batch_memory([c.shape for c in my_cells])
        need0 = sum(need) if need0 is None else need0
        if sum(need) <= FIT * avail:
            break
        e.close()
    else:
        bc, bj = choices[0]
        e = F.Engine(F.Config(device=local, precision=F.MIXED_PC))
        need, avail = e.batch_memory([c.shape for c in my_cells])
    smoother = ("node-block Jacobi" if bj else "point Jacobi") + (
        ", block PCG over the load cases" if bc else ", one PCG per load case")
    if (bc, bj) != choices[0] and sum(need) <= FIT * avail:
        smoother += f" (the defaults need {need0 / 1e9:.1f} GB, over one call's {FIT * avail / 1e9:.1f} GB)"
    e.batch(my_cells[:8], dLdC=W[:8], allow_unconverged=True)   # warm-up: library, autotuner code paths
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    t0 = time.perf_counter()
    try:
        C, infos, grads = e.batch(my_cells, dLdC=W, allow_unconverged=True)
    except F.FemhError as ex:   # the estimate fitted but the device did not: one-case PCG, FP32 directions
        if ex.code != F.FEMH_E_OOM or bc == 0:
            raise
        e.close()
        bc = 0
        smoother = ("node-block Jacobi" if bj else "point Jacobi") + ", one PCG per load case (block PCG ran out of memory)"
        e = F.Engine(F.Config(device=local, precision=F.MIXED_PC, block_cg=0, block_jacobi=bj))
        need, avail = e.batch_memory([c.shape for c in my_cells])
        e.batch(my_cells[:8], dLdC=W[:8], allow_unconverged=True)
        t0 = time.perf_counter()
        C, infos, grads = e.batch(my_cells, dLdC=W, allow_unconverged=True)
    t_batch = max_over_ranks(time.perf_counter() - t0, device="cuda")
    e.close()
    its = np.array([max(i["iterations"]) for i in infos])
    bad = int(max_over_ranks(sum(1 for i in infos if i["status"] != 0), device="cuda"))
    solve_s = max((i["solve_ms"] for i in infos), default=0.0) / 1e3   # device time of the solve proper
    out = {"cells": len(cells), "voxels": int(sum(c.size for c in cells)), "ranks": world,
           "cells_per_s": len(cells) / t_batch, "seconds": t_batch, "solve_seconds_rank0": solve_s,
           "calls_per_rank": int(max(1, np.ceil(sum(need) / (FIT * avail)))),
           "device_bytes_needed_rank0": float(sum(need)),
           "iterations_p50_p90_max_rank0": [int(np.percentile(its, 50)), int(np.percentile(its, 90)), int(its.max())],
           "not_converged_max_over_ranks": bad,
           "precision": "FP64 CG + FP32 multigrid, gradients contracted with a fixed dL/dC",
           "smoother": smoother,
           "set": "fields.uneven_batch(4096, seed=7)"}
    if rank == 0:
        e64 = F.Engine(F.Config(device=local, precision=F.FP64, block_jacobi=bj, block_cg=bc))
        k = min(fp64_sample, len(cells))
        e64.homogenize(cells[0])
        t0 = time.perf_counter()
        for c in cells[:k]:
            e64.homogenize(c, allow_unconverged=True)
            e64.grad(np.diag([1.0, 1.0, 1.0, 0.5, 0.5, 0.5]))
        t_one = (time.perf_counter() - t0) / k
        e64.close()
        out.update({"fp64_one_at_a_time_cells_per_s_one_gpu": 1.0 / t_one,
                    "fp64_sample": f"first {k} cells of the set, one femh_homogenize + femh_homogenize_grad each",
                    "speedup_per_gpu_vs_fp64_one_at_a_time": (len(cells) / t_batch / world) * t_one})
    return out


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
    Ct = target_tensor(n)

    stream = torch.cuda.current_stream()
    cfg = F.Config(device=local, precision=F.MIXED_PC, solver=F.GMG_PCG, autotune=0 if args.no_autotune else 1,
                   graph_chunk=0 if args.no_graphs else 8)
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
    traffic, traffic_note = kernel_traffic(top["name"])
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 preconditioner / f64 CG",
        "data": "synthetic (seeded filtered-noise densities)",
        "config": workload_config(n, world),
        "precision": "FP64 CG and operator, FP32 multigrid V-cycle (FP64 inner products and coarse solve)",
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
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic, "traffic_note": traffic_note,
                     "peak_kind": peak_kind, "share_of_step": top["total_ms"] / tot_ms,
                     "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms},
        "kernels": sorted(({"name": s["name"], "launches": s["launches"], "ms": round(s["total_ms"], 4),
                            "share": round(s["total_ms"] / tot_ms, 4)} for s in stats),
                          key=lambda d: -d["ms"])[:12],
    }
    eng.close()
    eng64.close()
    if not args.no_batch:
        out["batched_uneven"] = batched_uneven(F, local, args.batch_cells, world, rank)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(rho_h, Ct)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args, world, rank):
    """The reference path's CPU implementation on the host cores: the oracle
    port (the reference's own solver library, topoOptLib, is not in its tree),
    converged FP64 multigrid-PCG solves of the same workload, measured.  No GPU
    code runs.  Rank 0 alone runs and prints; other ranks exit without work.
    A full solve takes about a minute, so the timed steps stop once
    REFERENCE_BUDGET_S seconds are spent (at least one); `steps` reports the
    solves actually timed."""
    if rank != 0:
        return
    from fem_b200 import fields
    from oracle import oracle as O
    O.build()
    n = args.n
    rho = fields.smooth_cell(n, 4.0, seed=2)
    Ct = target_tensor(n)
    warm = min(args.warmup, 3)
    for _ in range(warm):   # page the library and the OpenMP pool in on a small cell
        O.mg_homogenize(fields.smooth_cell(32, 4.0, seed=2), tol=1e-10, want_chi=False, block=True)
    secs, cb = [], None
    t_start = time.perf_counter()
    while len(secs) < max(1, args.steps):
        cb = cpu_baseline(rho, Ct)
        secs.append(cb["seconds_per_tensor"])
        if time.perf_counter() - t_start > REFERENCE_BUDGET_S:
            break
    sec = statistics.median(secs)
    out = {
        "metric": METRIC, "value": 1.0 / sec, "unit": UNIT, "n_gpus": world, "steps": len(secs),
        "warmup": warm, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded filtered-noise densities)",
        "impl": "reference", "config": workload_config(n, world),
        "precision": "FP64 throughout (CPU)",
        "method": "the reference's: one multigrid PCG per load case (the GPU arm's V-cycle), no block CG",
        "timing": f"{len(secs)} full solve(s) timed (median), {warm} warm-up solve(s) of a 32^3 cell; "
                  f"requested --steps {args.steps} --warmup {args.warmup}",
        "cpu_baseline": {"value": 1.0 / sec, "unit": UNIT, "cores": cb["cores"], "kind": "port",
                         "sample": cb["sample"]},
        "e2e": {"value": 1.0 / sec, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def target_tensor(n: int) -> np.ndarray:
    """C_t = C^H of the independent seed-5 cell of the same size: from the
    committed FP64 fixture where it exists (128^3), else the CPU oracle."""
    path = os.path.join(ROOT, "tests", "golden", "large_cells.json")
    if os.path.exists(path):
        d = json.load(open(path))
        rec = d.get(f"c4_{n}")
        if rec:
            return np.array(rec["C_target"]).reshape(6, 6)
    from fem_b200 import fields
    from oracle import oracle as O
    return O.mg_homogenize(fields.smooth_cell(n, 4.0, seed=5), tol=1e-10, want_chi=False)[0]


REFERENCE_BUDGET_S = 150.0


if __name__ == "__main__":
    main()
