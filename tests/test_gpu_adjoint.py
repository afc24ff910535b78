"""Adjoint checks on the GPU (the 64^3 adjoint workload):
  * L = ||C^H - C_t||_F^2 with C_t the C^H of an independent seeded cell;
    dL/drho from the adjoint kernel against central finite differences of the
    full GPU solve at 64 randomly chosen voxels, h = 1e-6, FP64, rel <= 1e-5;
  * the same gradient against the restated reference formula (oracle) at 64^3;
  * the torch.autograd.Function binding passes torch.autograd.gradcheck.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL_GRAD = 1e-5


def test_adjoint_vs_central_differences_64(femh):
    from fem_b200 import fields
    n = 64
    rho = fields.smooth_cell(n, 4.0, seed=4)
    eng_t = femh.Engine(tol=1e-12)
    Ct, _ = eng_t.homogenize(fields.smooth_cell(n, 4.0, seed=5))
    eng = femh.Engine(tol=1e-12)
    C, _ = eng.homogenize(rho)
    g = eng.grad(2.0 * (C - Ct))
    rng = np.random.default_rng(6)
    picks = rng.choice(n ** 3, 64, replace=False)
    h = 1e-6
    fd = np.empty(64)
    an = np.empty(64)
    probe = femh.Engine(tol=1e-12)
    for t, flat in enumerate(picks):
        i = np.unravel_index(flat, rho.shape)
        rp = rho.copy(); rp[i] += h
        rm = rho.copy(); rm[i] -= h
        Lp = np.sum((probe.homogenize(rp)[0] - Ct) ** 2)
        Lm = np.sum((probe.homogenize(rm)[0] - Ct) ** 2)
        fd[t] = (Lp - Lm) / (2 * h)
        an[t] = g[i]
    # relative to the largest probed gradient (entries can be near zero)
    assert np.abs(fd - an).max() <= TOL_GRAD * np.abs(an).max()


def test_adjoint_vs_oracle_64(femh, oracle):
    from fem_b200 import fields
    n = 64
    rho = fields.smooth_cell(n, 4.0, seed=4)
    Ct = oracle.c_iso(0.05, 0.3)
    eng = femh.Engine(tol=1e-12)
    C, _ = eng.homogenize(rho)
    g = eng.grad(2.0 * (C - Ct))
    chi = eng.fluctuation()
    go = oracle.grad(rho, chi, 2.0 * (C - Ct))
    assert np.abs(g - go).max() <= TOL_GRAD * np.abs(go).max()


def test_torch_autograd_gradcheck(femh):
    import torch
    from fem_b200 import fields
    from fem_b200.autograd import homogenize
    eng = femh.Engine(tol=1e-13)
    rho = torch.tensor(fields.smooth_cell(4, 1.0, seed=8) * 0.6 + 0.3, dtype=torch.float64,
                       device="cuda", requires_grad=True)
    W = torch.randn(6, 6, dtype=torch.float64, device="cuda")

    def f(r):
        return (homogenize(r, eng) * W).sum()
    assert torch.autograd.gradcheck(f, (rho,), eps=1e-6, atol=1e-7, rtol=1e-5)


def test_field_chain_rule_on_device(femh):
    """femh_field_gradient: the field chain rule of FEM3DFun::df
    (fast_fem/FEM3DFun.cpp:252-266) for a piecewise-constant field, on the
    device -- equal to the per-voxel adjoint gradient summed over each
    parameter's voxels (plus the per-voxel density term), bit-identical
    across calls; voxels mapped to -1 contribute nothing; a parameter index out
    of range is an argument error."""
    from fem_b200 import fields
    rho = fields.smooth_cell(16, 2.0, seed=21)
    e = femh.Engine()
    C, _ = e.homogenize(rho)
    dLdC = 2.0 * (C - np.diag([0.1] * 3 + [0.03] * 3))
    g = e.grad(dLdC)
    i, j, k = np.meshgrid(*(np.arange(16) // 4,) * 3, indexing="ij")
    vp = (i * 4 + j) * 4 + k
    gp = e.field_grad(dLdC, vp, 64, add=0.01)
    want = (g + 0.01).reshape(4, 4, 4, 4, 4, 4).sum(axis=(1, 3, 5)).ravel()
    assert np.abs(gp - want).max() < 1e-12 * np.abs(want).max()
    assert np.array_equal(gp, e.field_grad(dLdC, vp, 64, add=0.01))
    vp2 = vp.copy()
    vp2[:, :, :8] = -1
    want2 = np.bincount(vp2[vp2 >= 0].ravel(), weights=(g + 0.01)[vp2 >= 0].ravel(), minlength=64)
    assert np.abs(e.field_grad(dLdC, vp2, 64, add=0.01) - want2).max() < 1e-12 * np.abs(want2).max()
    vp2[0, 0, 0] = 64
    with pytest.raises(femh.FemhError) as ex:
        e.field_grad(dLdC, vp2, 64)
    assert ex.value.code == femh.FEMH_E_ARG
