"""ctypes access to the reference's own code built by oracle/build_ref.sh into
oracle/_ref/ (TEST INFRASTRUCTURE ONLY; tests/ alone import this module).

* ``nc_coarsen``: SamplesGenerator's NumericalCoarsening::
  computeCoarsenedElasticityTensorAndParameters3D
  (SamplesGenerator/NumericalCoarsening.cpp:266-340), float as the reference
  ships it, PARDISO replaced by Eigen's sparse LU (oracle/ref_shim/pardiso_eigen.cpp).
* ``fastfem``: fast_fem's FEM3DFun setParam / f / df
  (fast_fem/FEM3DFun.cpp:128-268) over a PiecewiseConstant3D field, with the
  stand-in topoOptLib headers of oracle/ref_shim/ (its solve is the oracle's).

Each returns None when the library is absent (reference tree not present at
build time), so that the tests skip.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REF = os.path.join(_HERE, "_ref")
_libs: dict = {}

GENERAL, CUBIC, ORTHOTROPIC = 0, 1, 2


def _load(name):
    if name not in _libs:
        path = os.path.join(_REF, name)
        _libs[name] = ctypes.CDLL(path) if os.path.exists(path) else None
    return _libs[name]


def available(name: str) -> bool:
    return _load(name) is not None


def nc_coarsen(materials: np.ndarray, E, nu, densities, stype: int = CUBIC):
    """Reference outputs for one structure: (21 appended tensor values,
    appended parameters).  materials: int array [nx, ny, nz]."""
    L = _load("libnc_ref.so")
    if L is None:
        return None
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    L.ref_nc_coarsen3d.argtypes = [ctypes.c_int] * 3 + [ip, ctypes.c_int, dp, dp, dp, ctypes.c_int, dp, dp]
    L.ref_nc_coarsen3d.restype = ctypes.c_int
    nx, ny, nz = materials.shape
    m = np.ascontiguousarray(materials.ravel(), dtype=np.int32)
    E = np.ascontiguousarray(E, dtype=np.float64)
    nuv = np.ascontiguousarray(np.broadcast_to(np.asarray(nu, dtype=np.float64), E.shape))
    d = np.ascontiguousarray(densities, dtype=np.float64)
    tv, pv = np.zeros(21), np.zeros(16)
    k = L.ref_nc_coarsen3d(nx, ny, nz, m.ctypes.data_as(ip), len(E), E.ctypes.data_as(dp), nuv.ctypes.data_as(dp),
                           d.ctypes.data_as(dp), stype, tv.ctypes.data_as(dp), pv.ctypes.data_as(dp))
    if k < 0:
        raise RuntimeError(f"ref_nc_coarsen3d failed ({k})")
    return tv, pv[:k]


FIELD_PLAIN, FIELD_SYM, FIELD_CUBIC = 0, 1, 2


def field_index(kind: int, m: int, x) -> int:
    """The parameter the reference's field (kind: PiecewiseConstant3D /
    Sym3D / Cubic3D, m^3 parameters) assigns to the point x."""
    L = _load("libfastfem_ref.so")
    if L is None:
        return None
    L.ref_field_index.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 3
    L.ref_field_index.restype = ctypes.c_int
    return int(L.ref_field_index(kind, m, *[float(v) for v in x]))


def fastfem(n: int, x0: np.ndarray, nu: float, G0: np.ndarray, wG: np.ndarray, m0: float, mw: float,
            kind: int = FIELD_PLAIN):
    """The reference's FEM3DFun on an n^3 cell with an m^3 field of `kind`
    (x0 of m^3 parameters): dict of G (upper triangle, as the reference fills
    it), f, df (m^3), distribution (n^3), density, status."""
    L = _load("libfastfem_ref.so")
    if L is None:
        return None
    dp = ctypes.POINTER(ctypes.c_double)
    L.ref_ff_eval.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, dp, dp, ctypes.c_double,
                              ctypes.c_double, dp, dp, dp, dp, dp]
    L.ref_ff_eval.restype = ctypes.c_int
    x0 = np.ascontiguousarray(x0, dtype=np.float64).ravel()
    m = round(x0.size ** (1.0 / 3.0))
    assert m ** 3 == x0.size
    G0 = np.ascontiguousarray(G0, dtype=np.float64)
    wG = np.ascontiguousarray(wG, dtype=np.float64)
    G, f, df = np.zeros(36), np.zeros(1), np.zeros(m ** 3)
    dist, dens = np.zeros(n ** 3), np.zeros(1)
    st = L.ref_ff_eval(n, m, kind, nu, x0.ctypes.data_as(dp), G0.ctypes.data_as(dp), wG.ctypes.data_as(dp), m0, mw,
                       G.ctypes.data_as(dp), f.ctypes.data_as(dp), df.ctypes.data_as(dp),
                       dist.ctypes.data_as(dp), dens.ctypes.data_as(dp))
    return {"G": G.reshape(6, 6), "f": float(f[0]), "df": df, "distribution": dist.reshape(n, n, n),
            "density": float(dens[0]), "status": st}
