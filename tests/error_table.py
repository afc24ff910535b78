"""Per-entry error of the engine's C^H against the FP64 oracle (the checker), for
every precision mode, on the CPU parity workload (32^3 Bernoulli(0.5) binary
cell, seed 1, SIMP law with E_min = 1e-6: stiffness contrast 1e6) and a 16^3
smooth cell.  Prints a markdown table; needs a CUDA device.

    python tests/error_table.py > error_table.md
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import fem_b200 as F  # noqa: E402
from fem_b200 import fields  # noqa: E402
from oracle import oracle as O  # noqa: E402

MODES = (
    ("FP64 GMG-PCG", dict(precision=F.FP64)),
    ("FP64 Jacobi-PCG", dict(precision=F.FP64, solver=F.JACOBI_PCG)),
    ("mixed-PC", dict(precision=F.MIXED_PC)),
    ("mixed-PC bf16 p", dict(precision=F.MIXED_PC, store_bf16=1)),
    ("mixed DC", dict(precision=F.MIXED)),
    ("mixed DC bf16", dict(precision=F.MIXED, store_bf16=1)),
)
PAIRS = [(i, j) for i in range(6) for j in range(i + 1)]
NAMES = ["xx", "yy", "zz", "yz", "xz", "xy"]


def table(title, rho):
    Co = O.homogenize(rho)[0]
    scale = np.abs(Co).max()
    errs, iters = [], []
    for _, kw in MODES:
        C, info = F.Engine(F.Config(**kw)).homogenize(rho, allow_unconverged=True)
        errs.append(np.abs(C - Co) / scale)
        iters.append((max(info["iterations"]), info["outer_iterations"], max(info["rel_residual"]), info["status"]))
    print(f"### {title}\n")
    print("|C_IJ - C_IJ(oracle)| / max|C(oracle)| per lower-triangle entry (oracle: FP64 Jacobi-PCG to 1e-10)\n")
    print("| entry | oracle C_IJ | " + " | ".join(m for m, _ in MODES) + " |")
    print("|---|---:|" + "---:|" * len(MODES))
    for i, j in PAIRS:
        print(f"| {NAMES[i]}-{NAMES[j]} | {Co[i, j]:.6e} | " + " | ".join(f"{e[i, j]:.1e}" for e in errs) + " |")
    print("| max | | " + " | ".join(f"{e.max():.1e}" for e in errs) + " |")
    print("| CG iterations (max over load cases) / outer steps / residual / status | | "
          + " | ".join(f"{a} / {b} / {c:.1e} / {d}" for a, b, c, d in iters) + " |\n")


if __name__ == "__main__":
    table("32³ binary cell (Bernoulli 0.5, seed 1; the CPU parity workload)", fields.binary_cell(32, 0.5, seed=1))
    table("16³ smooth cell (filtered noise, sigma 2, seed 2)", fields.smooth_cell(16, sigma=2.0, seed=2))
