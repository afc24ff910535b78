"""Seeded synthetic density fields of the benchmark workloads.

No dataset ships with the reference for this path (its level*_matAssignments.bin
inputs, fast_fem/run3d.cpp:214, are absent), so seeded fields with the
workloads' shapes and value distributions stand in:

* ``binary_cell``   -- each voxel solid with probability p (32^3 parity case;
  per-cell volume fraction of the uneven batch);
* ``smooth_cell``   -- periodic white noise N(0,1), Gaussian filter of std
  sigma voxels (FFT, periodic), standardised to mean 0 / std 1, sigmoid with
  slope 4, mapped affinely onto [1e-3, 1] (128^3 plain and 64^3/128^3 adjoint
  workloads);
* ``median_cell``   -- the same filtered field with sigma = 8 thresholded at
  its median: binary, volume fraction 0.5 (256^3 mixed-precision workload);
* ``uneven_batch``  -- 4096 cells with n in {16,24,32,48,64} drawn with
  probabilities {.30,.25,.25,.15,.05}, binary voxels with a per-cell volume
  fraction ~ U[0.2, 0.6].
"""
from __future__ import annotations

import numpy as np


def _filtered(n: int, sigma: float, seed: int) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    z = rng.standard_normal((n, n, n))
    k = np.fft.fftfreq(n) * 2 * np.pi
    kx, ky, kz = np.meshgrid(k, k, k, indexing="ij")
    g = np.exp(-0.5 * sigma ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    f = np.real(np.fft.ifftn(np.fft.fftn(z) * g))
    return (f - f.mean()) / f.std()


def binary_cell(n: int, p: float = 0.5, seed: int = 1) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return (rng.random((n, n, n)) < p).astype(np.float64)


def smooth_cell(n: int, sigma: float = 4.0, seed: int = 2, slope: float = 4.0) -> np.ndarray:
    s = 1.0 / (1.0 + np.exp(-slope * _filtered(n, sigma, seed)))
    return np.ascontiguousarray(1e-3 + (1.0 - 1e-3) * s)


def median_cell(n: int, sigma: float = 8.0, seed: int = 3) -> np.ndarray:
    f = _filtered(n, sigma, seed)
    return np.ascontiguousarray((f > np.median(f)).astype(np.float64))


BATCH_SIZES = (16, 24, 32, 48, 64)
BATCH_PROBS = (0.30, 0.25, 0.25, 0.15, 0.05)


def uneven_batch(ncell: int = 4096, seed: int = 7, count: int | None = None):
    """The seeded uneven set; ``count`` returns only its first cells (the same
    draws as the full set)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ns = rng.choice(BATCH_SIZES, size=ncell, p=BATCH_PROBS)
    vf = rng.uniform(0.2, 0.6, size=ncell)
    cells = []
    for n, v in list(zip(ns, vf))[:ncell if count is None else count]:
        cells.append((rng.random((n, n, n)) < v).astype(np.float64))
    return cells
