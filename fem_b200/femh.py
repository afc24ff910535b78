"""Python binding of libfemh (ctypes over the C ABI in include/femh.h).

Thin by design: every numeric step runs in libfemh's CUDA kernels.  Loading
fails loudly when the library is missing; there is no CPU fallback.

Mirrors the reference's homogenization entry points (desaic/fem):
``Engine.homogenize`` <-> FEM3DFun::setParam's solve + energy loop
(fast_fem/FEM3DFun.cpp:128-196), ``Engine.grad`` <-> FEM3DFun::df
(fast_fem/FEM3DFun.cpp:222-268), ``Engine.full_field`` <-> copyPeriodicU
(fast_fem/FEM3DFun.cpp:31-56), ``Engine.batch`` <-> the sample generator's
per-cell loop (SamplesGenerator/SamplesGeneratorImpl.cpp:3703-3736).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field, fields
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfemh.so")

FEMH_OK, FEMH_E_ARG, FEMH_E_CUDA, FEMH_E_OOM, FEMH_E_NOT_CONVERGED, FEMH_E_BREAKDOWN, FEMH_E_STATE = range(7)
INTERP_SIMP, INTERP_RAMP3, INTERP_BINARY = 0, 1, 2
FP64, MIXED, MIXED_PC = 0, 1, 2
JACOBI_PCG, GMG_PCG = 0, 1

#: every exported symbol of include/femh.h
EXPORTS = (
    "femh_config_default", "femh_create", "femh_destroy", "femh_homogenize", "femh_homogenize_grad",
    "femh_dCdrho", "femh_force_tensors", "femh_full_field", "femh_fluctuation", "femh_apply_operator", "femh_homogenize_batch",
    "femh_last_error", "femh_set_stream", "femh_kernel_launches", "femh_profile", "femh_profile_read",
    "femh_energy_noalloc", "femh_batch_memory", "femh_field_gradient",
)


class FemhError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"femh error {code}: {msg}")
        self.code = code


class _Config(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int), ("interp", ctypes.c_int),
        ("E_s", ctypes.c_double), ("E_min", ctypes.c_double), ("penal", ctypes.c_double), ("nu", ctypes.c_double),
        ("bin_hi", ctypes.c_double), ("bin_lo", ctypes.c_double),
        ("rho_min", ctypes.c_double), ("rho_max", ctypes.c_double),
        ("precision", ctypes.c_int), ("solver", ctypes.c_int),
        ("pre_smooth", ctypes.c_int), ("post_smooth", ctypes.c_int),
        ("omega", ctypes.c_double), ("coarse_max_nodes", ctypes.c_int),
        ("tol", ctypes.c_double), ("max_iter", ctypes.c_int),
        ("inner_tol", ctypes.c_double), ("max_outer", ctypes.c_int),
        ("store_bf16", ctypes.c_int), ("graph_chunk", ctypes.c_int), ("coarse_avg", ctypes.c_int),
        ("autotune", ctypes.c_int), ("stencil_variant", ctypes.c_int), ("warm_start", ctypes.c_int),
        ("cheb_ratio", ctypes.c_double), ("block_jacobi", ctypes.c_int), ("block_cg", ctypes.c_int),
    ]


class _Info(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int), ("iterations", ctypes.c_int * 6), ("outer_iterations", ctypes.c_int),
        ("rel_residual", ctypes.c_double * 6), ("solve_ms", ctypes.c_double), ("density", ctypes.c_double),
    ]


class _Cell(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("h", ctypes.c_double),
                ("rho", ctypes.POINTER(ctypes.c_double))]


class _KStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 64), ("launches", ctypes.c_longlong), ("total_ms", ctypes.c_double),
                ("bytes", ctypes.c_double)]


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libfemh.so (build it with fem_b200/build.py first)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FemhError(FEMH_E_CUDA, f"{path} missing: run `python fem_b200/build.py` (no CPU fallback exists)")
    L = ctypes.CDLL(path)
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int
    L.femh_config_default.argtypes = [ctypes.POINTER(_Config)]
    L.femh_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(_Config)]
    L.femh_destroy.argtypes = [vp]
    L.femh_homogenize.argtypes = [vp, ip, ip, ip, ctypes.c_double, vp, ip, dp, ctypes.POINTER(_Info)]
    L.femh_homogenize_grad.argtypes = [vp, dp, vp, ip]
    L.femh_dCdrho.argtypes = [vp, vp, ip]
    L.femh_force_tensors.argtypes = [vp, vp]
    L.femh_full_field.argtypes = [vp, ip, vp, ip]
    L.femh_fluctuation.argtypes = [vp, vp, ip]
    L.femh_apply_operator.argtypes = [vp, ip, ip, ip, ctypes.c_double, vp, vp, vp, ip]
    L.femh_homogenize_batch.argtypes = [vp, ip, ctypes.POINTER(_Cell), dp, vp, vp, ctypes.POINTER(_Info)]
    L.femh_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    L.femh_set_stream.argtypes = [vp, vp]
    L.femh_kernel_launches.argtypes = [vp]
    L.femh_kernel_launches.restype = ctypes.c_longlong
    L.femh_profile.argtypes = [vp, ip]
    L.femh_profile_read.argtypes = [vp, ctypes.POINTER(_KStat), ip, ctypes.POINTER(ctypes.c_int)]
    L.femh_energy_noalloc.argtypes = [ctypes.POINTER(_Config), ip, ip, ip, ctypes.c_double, vp, vp, vp, vp]
    L.femh_batch_memory.argtypes = [vp, ip, ctypes.POINTER(_Cell), dp, dp]
    L.femh_field_gradient.argtypes = [vp, dp, ctypes.c_double, ip, ctypes.POINTER(ctypes.c_int), dp]
    _lib = L
    return L


@dataclass
class Config:
    """Engine configuration (fields of femh_config; defaults from femh_config_default)."""
    device: int = 0
    interp: int = INTERP_SIMP
    E_s: float = 1.0
    E_min: float = 1e-6
    penal: float = 3.0
    nu: float = 0.3
    bin_hi: float = 1.0
    bin_lo: float = 1e-4
    rho_min: float = 0.0
    rho_max: float = 1.0
    precision: int = FP64
    solver: int = GMG_PCG
    pre_smooth: int = 3
    post_smooth: int = 3
    omega: float = 0.35
    coarse_max_nodes: int = 64
    tol: float = 1e-10
    max_iter: int = 20000
    inner_tol: float = 1e-5
    max_outer: int = 8
    store_bf16: int = 0
    graph_chunk: int = 8
    coarse_avg: int = 0
    autotune: int = 1
    stencil_variant: int = 0
    warm_start: int = 0
    cheb_ratio: float = 64.0
    block_jacobi: int = 1
    block_cg: int = 1

    def to_c(self) -> _Config:
        c = _Config()
        for f in fields(self):
            setattr(c, f.name, getattr(self, f.name))
        return c


def _info_dict(i: _Info) -> dict:
    return {
        "status": i.status, "iterations": list(i.iterations), "outer_iterations": i.outer_iterations,
        "rel_residual": list(i.rel_residual), "solve_ms": i.solve_ms, "density": i.density,
    }


def _ptr(a) -> ctypes.c_void_p:
    """Host numpy array or device torch tensor -> (pointer, on_device)."""
    return ctypes.c_void_p(a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr())


def _is_dev(a) -> int:
    return 0 if isinstance(a, np.ndarray) else int(getattr(a, "is_cuda", False))


class Engine:
    """One libfemh handle (one CUDA stream)."""

    def __init__(self, config: Optional[Config] = None, **kw):
        self.lib = load_library()
        self.config = config if config is not None else Config(**kw)
        h = ctypes.c_void_p()
        st = self.lib.femh_create(ctypes.byref(h), ctypes.byref(self.config.to_c()))
        if st != FEMH_OK:
            raise FemhError(st, "femh_create failed (no CUDA device or bad config)")
        self.h = h
        self.shape = None
        self._ncells = 0   # cells of the last solve (their fields stay resident)

    def close(self):
        if getattr(self, "h", None):
            self.lib.femh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self, st: int):
        buf = ctypes.create_string_buffer(1024)
        self.lib.femh_last_error(self.h, buf, 1024)
        return FemhError(st, buf.value.decode())

    def _check(self, st: int, allow=(FEMH_OK,)):
        if st not in allow:
            raise self._err(st)
        return st

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.femh_kernel_launches(self.h))

    def profile(self, enable: bool = True):
        """Per-kernel CUDA-event timing (graphs off while enabled); clears stats."""
        self._check(self.lib.femh_profile(self.h, int(enable)))

    def profile_read(self) -> list[dict]:
        n = ctypes.c_int()
        self._check(self.lib.femh_profile_read(self.h, None, 0, ctypes.byref(n)))
        arr = (_KStat * max(n.value, 1))()
        self._check(self.lib.femh_profile_read(self.h, arr, n.value, ctypes.byref(n)))
        return [{"name": a.name.decode(), "launches": a.launches, "total_ms": a.total_ms, "bytes": a.bytes}
                for a in arr[:n.value]]

    def set_stream(self, stream_ptr: int | None):
        self._check(self.lib.femh_set_stream(self.h, ctypes.c_void_p(stream_ptr or 0)))

    # ------------------------------------------------------------ forward
    def homogenize(self, rho, h: float | None = None, allow_unconverged: bool = False):
        """C^H (6x6 numpy) and the solve info of one periodic cell.

        rho: (nx, ny, nz) float64 numpy array (host) or CUDA torch tensor."""
        self._autograd_rho = None
        nx, ny, nz = (int(s) for s in rho.shape)
        if isinstance(rho, np.ndarray):
            rho = np.ascontiguousarray(rho, dtype=np.float64)
        else:
            assert rho.dtype.__str__() == "torch.float64" and rho.is_contiguous()
        h = 1.0 / nx if h is None else float(h)
        C = np.zeros((6, 6))
        info = _Info()
        st = self.lib.femh_homogenize(self.h, nx, ny, nz, h, _ptr(rho), _is_dev(rho),
                                      C.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(info))
        allow = (FEMH_OK, FEMH_E_NOT_CONVERGED, FEMH_E_BREAKDOWN) if allow_unconverged else (FEMH_OK,)
        self._check(st, allow)
        self.shape = (nx, ny, nz)
        self._ncells = 1
        return C, _info_dict(info)

    def grad(self, dLdC, out=None):
        """dL/drho for dL/dC at the last solve (adjoint, no second solve)."""
        dLdC = np.ascontiguousarray(dLdC, dtype=np.float64).reshape(6, 6)
        if out is None:
            out = np.zeros(self.shape)
        self._check(self.lib.femh_homogenize_grad(self.h, dLdC.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                  _ptr(out), _is_dev(out)))
        return out

    def field_grad(self, dLdC, voxel_param, nparam: int, add: float = 0.0) -> np.ndarray:
        """Gradient w.r.t. the parameters of a piecewise-constant field
        (femh_field_gradient): voxel_param[i, j, k] = the parameter of that
        voxel (-1: none); ``add`` is added to dL/drho of every voxel."""
        dLdC = np.ascontiguousarray(dLdC, dtype=np.float64).reshape(6, 6)
        m = np.ascontiguousarray(voxel_param, dtype=np.int32).ravel()
        out = np.zeros(nparam)
        self._check(self.lib.femh_field_gradient(self.h, dLdC.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                 float(add), int(nparam),
                                                 m.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def dCdrho(self, out=None):
        """dC_IJ/drho_e for the 21 lower-triangle pairs: array [21, nx, ny, nz]."""
        if out is None:
            out = np.zeros((21,) + tuple(self.shape))
        self._check(self.lib.femh_dCdrho(self.h, _ptr(out), _is_dev(out)))
        return out

    def force_tensors(self):
        """femlib's force-driven coarse tensor (femh_force_tensors) of each
        cell of the last solve: [6, 6] after homogenize, [n, 6, 6] after batch."""
        if self._ncells < 1:
            raise FemhError(6, "call homogenize or batch first")
        out = np.zeros((self._ncells, 6, 6))
        self._check(self.lib.femh_force_tensors(self.h, _ptr(out)))
        return out[0] if self.shape is not None else out

    def full_field(self, load_case: int):
        nx, ny, nz = self.shape
        out = np.zeros((nx + 1, ny + 1, nz + 1, 3))
        self._check(self.lib.femh_full_field(self.h, int(load_case), _ptr(out), 0))
        return out

    def fluctuation(self):
        out = np.zeros((6,) + tuple(self.shape) + (3,))
        self._check(self.lib.femh_fluctuation(self.h, _ptr(out), 0))
        return out

    def apply_operator(self, rho, u, h: float | None = None):
        """y = K(rho) u for u of shape (6, nx, ny, nz, 3) (host float64)."""
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        nx, ny, nz = rho.shape
        assert u.shape == (6, nx, ny, nz, 3)
        y = np.zeros_like(u)
        h = 1.0 / nx if h is None else float(h)
        self._check(self.lib.femh_apply_operator(self.h, nx, ny, nz, h, _ptr(rho), _ptr(u), _ptr(y), 0))
        self.shape = None
        self._ncells = 0
        return y

    def batch_memory(self, shapes: Sequence[tuple]) -> tuple[list[float], float]:
        """Device bytes a batch call needs for each cell shape, and the bytes
        available to it (femh_batch_memory)."""
        need, avail = [], ctypes.c_double()
        for i, (nx, ny, nz) in enumerate(shapes):
            c = _Cell()
            c.nx, c.ny, c.nz, c.h = int(nx), int(ny), int(nz), 1.0
            b = ctypes.c_double()
            self._check(self.lib.femh_batch_memory(self.h, 1, ctypes.byref(c), ctypes.byref(b),
                                                   ctypes.byref(avail) if i == 0 else None))
            need.append(b.value)
        return need, avail.value

    def batch(self, rhos: Sequence[np.ndarray], h: float | None = None, dLdC=None, allow_unconverged=False,
              max_nodes: int | None = None):
        """Many cells in one set of launches.  Returns (C [n,6,6], infos, dLdrho list or None).

        The cells go to the engine in consecutive calls (at least one cell per
        call) of at most ``max_nodes`` voxels each, or by default of what fits
        the device (femh_batch_memory's estimate against 92% of the memory
        available; the whole set when it fits).  After a split call
        force_tensors() is not available (the engine holds only the last
        part's fields)."""
        sizes = [int(np.prod(r.shape)) for r in rhos]
        if max_nodes is None:
            need, avail = self.batch_memory([r.shape for r in rhos])
            cost, budget = need, 0.92 * avail
        else:
            cost, budget = sizes, max_nodes
        if sum(cost) > budget:
            dl = None if dLdC is None else np.ascontiguousarray(dLdC, dtype=np.float64).reshape(len(rhos), 6, 6)
            Cs, infos, grads = [], [], ([] if dLdC is not None else None)
            i = 0
            while i < len(rhos):
                j, used = i, 0.0
                while j < len(rhos) and (j == i or used + cost[j] <= budget):
                    used += cost[j]
                    j += 1
                C, inf, g = self._batch1(rhos[i:j], h, None if dl is None else dl[i:j], allow_unconverged)
                Cs.append(C)
                infos += inf
                if grads is not None:
                    grads += g
                i = j
            self._ncells = 0
            return np.concatenate(Cs), infos, grads
        return self._batch1(rhos, h, dLdC, allow_unconverged)

    def _batch1(self, rhos, h, dLdC, allow_unconverged):
        n = len(rhos)
        rhos = [np.ascontiguousarray(r, dtype=np.float64) for r in rhos]
        cells = (_Cell * n)()
        for i, r in enumerate(rhos):
            cells[i].nx, cells[i].ny, cells[i].nz = r.shape
            cells[i].h = (1.0 / r.shape[0]) if h is None else h
            cells[i].rho = r.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        C = np.zeros((n, 6, 6))
        infos = (_Info * n)()
        g = None
        gp = ctypes.c_void_p(0)
        dp = ctypes.c_void_p(0)
        if dLdC is not None:
            dLdC = np.ascontiguousarray(dLdC, dtype=np.float64).reshape(n, 6, 6)
            g = np.zeros(sum(r.size for r in rhos))
            gp = _ptr(g)
            dp = _ptr(dLdC)
        st = self.lib.femh_homogenize_batch(self.h, n, cells, C.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                            dp, gp, infos)
        allow = (FEMH_OK, FEMH_E_NOT_CONVERGED, FEMH_E_BREAKDOWN) if allow_unconverged else (FEMH_OK,)
        self._check(st, allow)
        self.shape = None
        self._ncells = n
        grads = None
        if g is not None:
            grads, o = [], 0
            for r in rhos:
                grads.append(g[o:o + r.size].reshape(r.shape))
                o += r.size
        return C, [_info_dict(i) for i in infos], grads
