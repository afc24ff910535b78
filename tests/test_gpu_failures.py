"""Failure detection through the C ABI, in the forms this engine can show
without faulting the GPU (every error path ends in a status the host reads):

* bad input: a NaN, infinite or negative density is an argument error
  (FEMH_E_ARG) before any solve, and the handle stays usable;
* an unconverged solve (max_iter reached) returns FEMH_E_NOT_CONVERGED with
  C^H and the residuals written;
* a bounded stage wait of the bulk-copy staged kernels that runs out: with
  FEMH_STAGE_WAIT_LIMIT=0 every stage wait gives up at once although its
  copies complete; the kernel drains its copies with the full limit, sets the
  handle's error flag and returns, the call reports FEMH_E_CUDA, and a fresh
  handle in the same process solves correctly;
* a device allocation that fails: FEMH_ARENA_LIMIT_BYTES caps a handle's
  set-up memory, the call reports FEMH_E_OOM, and a handle without the cap
  solves correctly;
* a block PCG whose preconditioner is not positive definite (a damped-Jacobi
  smoother with omega far above 2 / lambda_max): the block stops at its first
  check and the cell is solved again one load case at a time, where the
  one-case PCG falls back to Jacobi; the result is the one-case run's.
The reference has no error reporting on this path beyond fem_error and printed
PARDISO codes (femlib/include/femError.hpp:1-7, StepperCPU/src/pardiso_sym.cpp:60-68).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.fixture(scope="module")
def cell16():
    from fem_b200 import fields
    return fields.binary_cell(16, 0.5, seed=11)


@pytest.fixture(scope="module")
def ref16(oracle, cell16):
    return oracle.homogenize(cell16, tol=1e-12)[0]


@pytest.mark.parametrize("bad", [np.nan, np.inf, -0.25])
def test_bad_density_is_an_argument_error(femh, cell16, ref16, bad):
    e = femh.Engine()
    rho = cell16.copy()
    rho[3, 4, 5] = bad
    with pytest.raises(femh.FemhError) as ex:
        e.homogenize(rho)
    assert ex.value.code == femh.FEMH_E_ARG and "density" in str(ex.value)
    with pytest.raises(femh.FemhError) as ex2:   # the gradient needs a successful solve
        e.grad(np.eye(6), out=np.zeros(cell16.shape))
    assert ex2.value.code == femh.FEMH_E_STATE
    C, info = e.homogenize(cell16)   # the same handle, good input
    assert info["status"] == 0 and _rel(C, ref16) < 1e-8


def test_bad_density_in_a_batch(femh, cell16):
    e = femh.Engine(precision=femh.MIXED_PC)
    rho = cell16.copy()
    rho[0, 0, 1] = np.nan
    with pytest.raises(femh.FemhError) as ex:
        e.batch([cell16, rho])
    assert ex.value.code == femh.FEMH_E_ARG


def test_max_iter_reached_reports_not_converged(femh, cell16, ref16):
    e = femh.Engine(max_iter=3)
    lib = e.lib
    import ctypes
    C = np.zeros((6, 6))
    info = femh.femh._Info()
    rho = np.ascontiguousarray(cell16)
    st = lib.femh_homogenize(e.h, 16, 16, 16, 1.0 / 16, ctypes.c_void_p(rho.ctypes.data), 0,
                             C.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(info))
    assert st == femh.FEMH_E_NOT_CONVERGED and info.status == femh.FEMH_E_NOT_CONVERGED
    assert max(info.iterations) <= 3 + 8   # whole captured graph chunks
    assert min(info.rel_residual) > 1e-10 and np.all(np.isfinite(list(info.rel_residual)))
    # results are written: a partly converged C^H, already close to the answer
    assert np.all(np.isfinite(C)) and 1e-8 < _rel(C, ref16) < 0.5
    C2, info2 = e.homogenize(cell16, allow_unconverged=True)
    assert info2["status"] == femh.FEMH_E_NOT_CONVERGED and np.array_equal(C, C2)


def test_stage_wait_timeout_reports_cuda_error(femh, cell16, ref16, monkeypatch):
    import torch
    monkeypatch.setenv("FEMH_STAGE_WAIT_LIMIT", "0")
    e = femh.Engine(stencil_variant=6, autotune=0, max_iter=40)   # FP64 bulk-copy staged kernel
    monkeypatch.delenv("FEMH_STAGE_WAIT_LIMIT")
    with pytest.raises(femh.FemhError) as ex:
        e.homogenize(cell16)
    assert ex.value.code == femh.FEMH_E_CUDA and "timed out" in str(ex.value)
    e.close()
    torch.cuda.synchronize()   # the context is intact
    f = femh.Engine(stencil_variant=6, autotune=0)
    C, info = f.homogenize(cell16)
    assert info["status"] == 0 and _rel(C, ref16) < 1e-8


def test_allocation_failure_reports_oom(femh, cell16, ref16, monkeypatch):
    monkeypatch.setenv("FEMH_ARENA_LIMIT_BYTES", str(1 << 20))
    e = femh.Engine()
    monkeypatch.delenv("FEMH_ARENA_LIMIT_BYTES")
    with pytest.raises(femh.FemhError) as ex:
        e.homogenize(cell16)
    assert ex.value.code == femh.FEMH_E_OOM
    f = femh.Engine()
    C, info = f.homogenize(cell16)
    assert info["status"] == 0 and _rel(C, ref16) < 1e-8


def test_indefinite_block_falls_back_to_one_case_pcg(femh, cell16, ref16):
    """omega = 1.9 without Chebyshev weights makes every sweep amplify the
    high-frequency error, so the V-cycle is indefinite and z.r of the start is
    not positive: the block reports CG_BLOCK_FAIL at once and the host solves
    the cell one load case at a time (FP64, the same kernel layouts: the very
    computation of block_cg=0, the same iteration counts and C^H)."""
    kw = dict(precision=femh.FP64, omega=1.9, cheb_ratio=0.0, pre_smooth=2, post_smooth=2, max_iter=5000,
              autotune=0)
    Cb, ib = femh.Engine(block_cg=1, **kw).homogenize(cell16)
    Cc, ic = femh.Engine(block_cg=0, **kw).homogenize(cell16)
    assert ib["status"] == 0 and max(ib["rel_residual"]) < 1e-10
    assert ib["iterations"] == ic["iterations"]
    assert _rel(Cb, Cc) < 1e-13
    assert _rel(Cb, ref16) < 1e-8
