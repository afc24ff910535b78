"""ctypes wrapper of the CPU FP64 oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module; the engine in ``fem_b200`` never does.  Every function follows the
C restatement in ``femh_oracle.c``, whose header lists the reference lines each
piece restates.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libfemh_oracle.so")
_lib = None

INTERP_SIMP, INTERP_RAMP3, INTERP_BINARY = 0, 1, 2


class Material(ctypes.Structure):
    _fields_ = [
        ("interp", ctypes.c_int),
        ("E_s", ctypes.c_double),
        ("E_min", ctypes.c_double),
        ("penal", ctypes.c_double),
        ("nu", ctypes.c_double),
        ("bin_hi", ctypes.c_double),
        ("bin_lo", ctypes.c_double),
    ]


def material(interp=INTERP_SIMP, E_s=1.0, E_min=1e-6, penal=3.0, nu=0.3, bin_hi=1.0, bin_lo=1e-4):
    return Material(interp, E_s, E_min, penal, nu, bin_hi, bin_lo)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    srcs = [os.path.join(_HERE, f) for f in ("femh_oracle.c", "femh_oracle_mg.c", "femh_oracle.h", "Makefile")]
    if force or not os.path.exists(_LIB_PATH) or any(os.path.getmtime(_LIB_PATH) < os.path.getmtime(f) for f in srcs):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.fo_k0.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, dp]
        L.fo_coef.argtypes = [ctypes.POINTER(Material), ctypes.c_double]
        L.fo_coef.restype = ctypes.c_double
        L.fo_dcoef.argtypes = [ctypes.POINTER(Material), ctypes.c_double]
        L.fo_dcoef.restype = ctypes.c_double
        L.fo_apply.argtypes = [ctypes.c_int] * 3 + [dp, dp, dp, dp, ctypes.c_int]
        L.fo_rhs.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, dp, dp, dp]
        L.fo_inv_diag.argtypes = [ctypes.c_int] * 3 + [dp, dp, dp]
        L.fo_energy.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, dp, dp, dp, dp]
        L.fo_dCdrho.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, dp, ctypes.POINTER(Material), dp, dp, dp]
        L.fo_grad.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, dp, ctypes.POINTER(Material), dp, dp, dp, dp]
        L.fo_homogenize.argtypes = [ctypes.c_int] * 3 + [
            ctypes.c_double, dp, ctypes.POINTER(Material), ctypes.c_double, ctypes.c_int,
            dp, dp, ctypes.POINTER(ctypes.c_int), dp]
        L.fo_homogenize.restype = ctypes.c_int
        L.fo_num_threads.restype = ctypes.c_int
        L.fo_pcg1.argtypes = [ctypes.c_int] * 3 + [dp, dp, dp, dp, dp, ctypes.c_double, ctypes.c_int, dp]
        L.fo_pcg1.restype = ctypes.c_int
        L.fo_mg_homogenize.argtypes = [ctypes.c_int] * 3 + [
            ctypes.c_double, dp, ctypes.POINTER(Material), ctypes.c_double, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_double, ctypes.c_int, dp, dp, ctypes.POINTER(ctypes.c_int), dp]
        L.fo_mg_homogenize.restype = ctypes.c_int
        L.fo_mg_homogenize_b.argtypes = [ctypes.c_int] * 3 + [
            ctypes.c_double, dp, ctypes.POINTER(Material), ctypes.c_double, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, dp, dp, ctypes.POINTER(ctypes.c_int), dp]
        L.fo_mg_homogenize_b.restype = ctypes.c_int
        L.fo_mg_apply.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, dp, ctypes.c_double, dp, dp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def k0(E=1.0, nu=0.3, h=1.0) -> np.ndarray:
    K = np.zeros((24, 24))
    lib().fo_k0(E, nu, h, _p(K))
    return K


def coef(mat: Material, rho: np.ndarray) -> np.ndarray:
    L = lib()
    return np.array([L.fo_coef(ctypes.byref(mat), float(r)) for r in np.ravel(rho)])


def apply(shape, K0: np.ndarray, c: np.ndarray, u: np.ndarray) -> np.ndarray:
    """y = K(c) u for u of shape [nrhs, nx, ny, nz, 3]."""
    nx, ny, nz = shape
    u = np.ascontiguousarray(u, dtype=np.float64)
    nrhs = u.size // (3 * nx * ny * nz)
    y = np.zeros_like(u)
    lib().fo_apply(nx, ny, nz, _p(np.ascontiguousarray(K0)), _p(np.ascontiguousarray(c, dtype=np.float64)),
                   _p(u), _p(y), nrhs)
    return y


def rhs(shape, h, K0, c) -> np.ndarray:
    nx, ny, nz = shape
    b = np.zeros((6, nx, ny, nz, 3))
    lib().fo_rhs(nx, ny, nz, h, _p(np.ascontiguousarray(K0)), _p(np.ascontiguousarray(c, dtype=np.float64)), _p(b))
    return b


def homogenize(rho: np.ndarray, h: float | None = None, mat: Material | None = None,
               tol: float = 1e-10, max_iter: int = 20000):
    """Returns (C[6,6], chi[6,nx,ny,nz,3], iters[6], rel[6], status)."""
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    nx, ny, nz = rho.shape
    if h is None:
        h = 1.0 / nx
    if mat is None:
        mat = material()
    C = np.zeros((6, 6))
    chi = np.zeros((6, nx, ny, nz, 3))
    iters = (ctypes.c_int * 6)()
    rel = np.zeros(6)
    st = lib().fo_homogenize(nx, ny, nz, h, _p(rho), ctypes.byref(mat), tol, max_iter,
                             _p(C), _p(chi), iters, _p(rel))
    return C, chi, list(iters), rel, st


def mg_homogenize(rho: np.ndarray, h: float | None = None, mat: Material | None = None,
                  tol: float = 1e-10, max_iter: int = 2000, pre: int = 3, post: int = 3,
                  cheb_ratio: float = 64.0, coarse_max: int = 64, want_chi: bool = True, block: bool = False):
    """Same problem and outputs as ``homogenize``, solved by the multigrid PCG of
    femh_oracle_mg.c (point-Jacobi sweeps, or node-block Jacobi with block).
    Returns (C[6,6], chi[6,nx,ny,nz,3] or None, iters[6], rel[6], status)."""
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    nx, ny, nz = rho.shape
    if h is None:
        h = 1.0 / nx
    if mat is None:
        mat = material()
    C = np.zeros((6, 6))
    chi = np.zeros((6, nx, ny, nz, 3)) if want_chi else None
    iters = (ctypes.c_int * 6)()
    rel = np.zeros(6)
    st = lib().fo_mg_homogenize_b(nx, ny, nz, h, _p(rho), ctypes.byref(mat), tol, max_iter, pre, post,
                                  cheb_ratio, coarse_max, 1 if block else 0, _p(C), _p(chi) if want_chi else None,
                                  iters, _p(rel))
    return C, chi, list(iters), rel, st


def mg_apply(shape, c: np.ndarray, u: np.ndarray, h: float = 1.0, nu: float = 0.3) -> np.ndarray:
    """y = K(c) u (six load cases, [6, nx, ny, nz, 3]) through the multigrid
    file's Hadamard-form apply; the rows of node 0 come back 0 (pinned)."""
    nx, ny, nz = shape
    u = np.ascontiguousarray(u, dtype=np.float64)
    y = np.zeros_like(u)
    lib().fo_mg_apply(nx, ny, nz, h, _p(np.ascontiguousarray(c, dtype=np.float64)), nu, _p(u), _p(y))
    return y


def energy(rho, chi, h=None, mat=None) -> np.ndarray:
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    nx, ny, nz = rho.shape
    h = 1.0 / nx if h is None else h
    mat = material() if mat is None else mat
    K0 = k0(1.0, mat.nu, h)
    c = coef(mat, rho)
    C = np.zeros((6, 6))
    lib().fo_energy(nx, ny, nz, h, _p(K0), _p(c), _p(np.ascontiguousarray(chi)), _p(C))
    return C


def dCdrho(rho, chi, h=None, mat=None) -> np.ndarray:
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    nx, ny, nz = rho.shape
    h = 1.0 / nx if h is None else h
    mat = material() if mat is None else mat
    K0 = k0(1.0, mat.nu, h)
    out = np.zeros((21, nx, ny, nz))
    lib().fo_dCdrho(nx, ny, nz, h, _p(K0), ctypes.byref(mat), _p(rho), _p(np.ascontiguousarray(chi)), _p(out))
    return out


def grad(rho, chi, dLdC, h=None, mat=None) -> np.ndarray:
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    nx, ny, nz = rho.shape
    h = 1.0 / nx if h is None else h
    mat = material() if mat is None else mat
    K0 = k0(1.0, mat.nu, h)
    out = np.zeros((nx, ny, nz))
    lib().fo_grad(nx, ny, nz, h, _p(K0), ctypes.byref(mat), _p(rho), _p(np.ascontiguousarray(chi)),
                  _p(np.ascontiguousarray(dLdC, dtype=np.float64)), _p(out))
    return out


def time_pcg(rho, iters: int, mat: Material | None = None, h: float | None = None) -> float:
    """Seconds per Jacobi-PCG iteration of all six load cases (FP64, OpenMP),
    measured over `iters` iterations of each load case at the full size."""
    import time
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    nx, ny, nz = rho.shape
    h = 1.0 / nx if h is None else h
    mat = material() if mat is None else mat
    K0 = k0(1.0, mat.nu, h)
    c = np.ascontiguousarray(coef(mat, rho))
    b = rhs(rho.shape, h, K0, c)
    dinv = np.zeros(rho.shape + (3,))
    L = lib()
    L.fo_inv_diag(nx, ny, nz, _p(K0), _p(c), _p(dinv))
    x = np.zeros(rho.shape + (3,))
    rel = np.zeros(1)
    t0 = time.perf_counter()
    for I in range(6):
        L.fo_pcg1(nx, ny, nz, _p(K0), _p(c), _p(dinv), _p(np.ascontiguousarray(b[I])), _p(x), 0.0, iters, _p(rel))
    return (time.perf_counter() - t0) / iters


def num_threads() -> int:
    return lib().fo_num_threads()


# ---------------------------------------------------------------- closed forms
def c_iso(E: float, nu: float) -> np.ndarray:
    """Isotropic Voigt stiffness (xx,yy,zz,yz,xz,xy; engineering shear)."""
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[[0, 1, 2], [0, 1, 2]] += 2 * mu
    C[3, 3] = C[4, 4] = C[5, 5] = mu
    return C


def c_laminate(Es, nu: float, axis: int = 2) -> np.ndarray:
    """Exact effective stiffness of a periodic stack of equal-thickness isotropic
    layers with moduli ``Es`` and Poisson ratio ``nu``, stacked along ``axis``.
    Classical laminate averaging: traction components continuous, in-plane
    strains continuous."""
    # Voigt components normal-coupled ("n") and in-plane ("p") for axis
    if axis == 2:
        n_idx, p_idx = [2, 3, 4], [0, 1, 5]
    elif axis == 1:
        n_idx, p_idx = [1, 3, 5], [0, 2, 4]
    else:
        n_idx, p_idx = [0, 4, 5], [1, 2, 3]
    Ann = np.zeros((3, 3)); Anp = np.zeros((3, 3)); App = np.zeros((3, 3))
    Bpn = np.zeros((3, 3))
    for E in Es:
        C = c_iso(E, nu)
        Cnn = C[np.ix_(n_idx, n_idx)]; Cnp = C[np.ix_(n_idx, p_idx)]
        Cpn = C[np.ix_(p_idx, n_idx)]; Cpp = C[np.ix_(p_idx, p_idx)]
        inv = np.linalg.inv(Cnn)
        Ann += inv; Anp += inv @ Cnp
        Bpn += Cpn @ inv; App += Cpp - Cpn @ inv @ Cnp
    m = len(Es)
    Ann /= m; Anp /= m; Bpn /= m; App /= m
    Snn = np.linalg.inv(Ann)            # sigma_n = Snn (eps_n + Anp eps_p)
    Ceff = np.zeros((6, 6))
    Ceff[np.ix_(n_idx, n_idx)] = Snn
    Ceff[np.ix_(n_idx, p_idx)] = Snn @ Anp
    Ceff[np.ix_(p_idx, n_idx)] = Bpn @ Snn
    Ceff[np.ix_(p_idx, p_idx)] = Bpn @ Snn @ Anp + App
    return Ceff
