"""GPU test of femh_energy_noalloc, the entry point for callers that cannot
call cudaMalloc (their device memory belongs to another allocator, or they
cannot afford cudaMalloc's implicit synchronisation): it must give the same
C^H as femh_homogenize for the fluctuation that solve produced, on two calls
in a row that reuse its fixed scratch array, and reject oversized cells.

The file name makes pytest collect it last, so a run that stops at the first
failure has already run every other test; it also passes alone in a fresh
process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-8   # the FP64 parity bar used by the other GPU tests


def _call(lib, cfg, shape, h, rho_d, chi_d, C_d, stream):
    nx, ny, nz = shape
    return lib.femh_energy_noalloc(ctypes.byref(cfg), nx, ny, nz, h, ctypes.c_void_p(rho_d.data_ptr()),
                                   ctypes.c_void_p(chi_d.data_ptr()), ctypes.c_void_p(C_d.data_ptr()),
                                   ctypes.c_void_p(stream))


def test_noalloc_energy_matches_homogenize(femh):
    import torch
    from fem_b200 import fields
    lib = femh.load_library()
    for n, seed in ((24, 3), (16, 8)):
        rho = fields.smooth_cell(n, 2.0, seed=seed)
        eng = femh.Engine()
        C_ref, info = eng.homogenize(rho)
        chi_d = torch.zeros((6, n, n, n, 3), dtype=torch.float64, device="cuda")
        eng._check(lib.femh_fluctuation(eng.h, ctypes.c_void_p(chi_d.data_ptr()), 1))
        rho_d = torch.from_numpy(rho).cuda()
        cfg = eng.config.to_c()
        cfg.device = torch.cuda.current_device()
        stream = torch.cuda.current_stream().cuda_stream
        for _ in range(2):   # two calls in a row share the scratch array
            C_d = torch.full((36,), float("nan"), dtype=torch.float64, device="cuda")
            assert _call(lib, cfg, (n, n, n), 1.0 / n, rho_d, chi_d, C_d, stream) == 0
            torch.cuda.synchronize()
            C = C_d.cpu().numpy().reshape(6, 6)
            assert np.abs(C - C_ref).max() < TOL_FP64 * np.abs(C_ref).max()
        eng.close()


def test_noalloc_rejects_oversized_cell(femh):
    import torch
    lib = femh.load_library()
    cfg = femh.Config(device=torch.cuda.current_device()).to_c()
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert _call(lib, cfg, (257, 256, 256), 1.0 / 256, dummy, dummy, dummy, 0) == 1   # FEMH_E_ARG
