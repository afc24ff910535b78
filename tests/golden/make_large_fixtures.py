"""Generates tests/golden/large_cells.json: C^H and dL/drho of the benchmark
workloads at their full sizes, computed by the CPU FP64 oracle's multigrid PCG
(oracle/femh_oracle_mg.c) to a relative residual of 1e-12.

The GPU tests (tests/test_gpu_fixtures.py) regenerate the same seeded fields
with fem_b200/fields.py and compare the engine's results with these numbers:

  c2_128    128^3 smooth cell (sigma 4, seed 2): C^H
  c3_256    256^3 median-thresholded binary cell (sigma 8, seed 3): C^H
  c4_64     64^3 smooth cell (seed 4) with the target C_t = C^H of the seed-5
  c4_128    cell of the same size; L = ||C - C_t||_F^2; dL/drho at 64 voxels
            drawn with seed 6 (central differences of the GPU solve check the
            same voxels), plus sum and sum of squares of the whole gradient
  c5_64     the first 64 cells of the seeded 4096-cell uneven set (seed 7):
            C^H of each

Each field also records sum(rho) so that a change of the field generator shows
up as a fixture mismatch rather than a solver error.  Runs on the host cores
(about an hour on 8 cores, 256^3 dominating); the committed JSON is what the
tests read.

usage: python tests/golden/make_large_fixtures.py [name ...]
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fem_b200 import fields  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "large_cells.json")
TOL = 1e-12


def solve(rho, chi=False):
    t = time.time()
    C, x, it, rel, st = O.mg_homogenize(rho, tol=TOL, max_iter=50000, want_chi=chi)
    assert st == 0, (st, it, rel)
    print(f"  {rho.shape} iterations {it} in {time.time() - t:.1f} s", flush=True)
    return C, x, it


def c2():
    rho = fields.smooth_cell(128, 4.0, seed=2)
    C, _, it = solve(rho)
    return {"field": "smooth_cell(128, 4.0, seed=2)", "rho_sum": float(rho.sum()), "C": C.ravel().tolist(),
            "iterations": it}


def c3():
    rho = fields.median_cell(256, 8.0, seed=3)
    C, _, it = solve(rho)
    return {"field": "median_cell(256, 8.0, seed=3)", "rho_sum": float(rho.sum()), "C": C.ravel().tolist(),
            "iterations": it}


def c4(n):
    rho = fields.smooth_cell(n, 4.0, seed=4)
    Ct, _, _ = solve(fields.smooth_cell(n, 4.0, seed=5))
    C, chi, it = solve(rho, chi=True)
    g = O.grad(rho, chi, 2.0 * (C - Ct)).ravel()
    rng = np.random.Generator(np.random.PCG64(6))
    vox = np.sort(rng.choice(rho.size, size=64, replace=False))
    return {"field": f"smooth_cell({n}, 4.0, seed=4)", "target_field": f"smooth_cell({n}, 4.0, seed=5)",
            "rho_sum": float(rho.sum()), "C": C.ravel().tolist(), "C_target": Ct.ravel().tolist(),
            "iterations": it, "loss": float(((C - Ct) ** 2).sum()), "voxels": vox.tolist(),
            "dLdrho": g[vox].tolist(), "dLdrho_sum": float(g.sum()), "dLdrho_sumsq": float((g * g).sum())}


def c5():
    cells = fields.uneven_batch(4096, seed=7, count=64)
    out = []
    for rho in cells:
        C, _, it = solve(rho)
        out.append({"n": int(rho.shape[0]), "rho_sum": float(rho.sum()), "C": C.ravel().tolist(),
                    "iterations": it})
    return {"set": "fields.uneven_batch(4096, seed=7, count=64)", "cells": out}


JOBS = {"c2_128": c2, "c4_64": lambda: c4(64), "c4_128": lambda: c4(128), "c5_64": c5, "c3_256": c3}


def main(names):
    data = json.load(open(OUT)) if os.path.exists(OUT) else {}
    data["generator"] = "tests/golden/make_large_fixtures.py"
    data["oracle"] = f"oracle/femh_oracle_mg.c multigrid PCG, FP64, relative residual {TOL}"
    for name in names or list(JOBS):
        print(name, flush=True)
        data[name] = JOBS[name]()
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main(sys.argv[1:])
