"""The benchmark workloads at their full sizes against the CPU FP64 oracle
(tests/golden/large_cells.json, made by tests/golden/make_large_fixtures.py
with the oracle's multigrid PCG to a relative residual of 1e-12), through the
C ABI:

  128^3 smooth cell            C^H, plain FP64 (1e-8) and mixed (1e-6)
  256^3 median-binary cell     C^H, plain FP64 (1e-8) and mixed (1e-6)
  64^3 / 128^3 smooth cells    C^H and dL/drho of ||C - C_t||_F^2 at 64 seeded
                               voxels (1e-5 of the largest of them), plus the
                               sum and sum of squares of the whole gradient
  64 cells of the uneven set   C^H of each cell from one batched call, FP64
                               (1e-8) and mixed (1e-6)

Tolerances are relative to the largest entry of the reference tensor (or
gradient).  Each field is regenerated from its seed; its recorded sum guards
against a change of the generator.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL_FP64, TOL_MIXED, TOL_GRAD = 1e-8, 1e-6, 1e-5
DATA = json.load(open(os.path.join(ROOT, "tests", "golden", "large_cells.json")))


def _need(key):
    if key not in DATA:
        pytest.skip(f"{key} not in tests/golden/large_cells.json")
    return DATA[key]


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


def _modes(femh):
    return [(femh.FP64, TOL_FP64), (femh.MIXED_PC, TOL_MIXED)]


def test_c2_128_smooth_cell(femh):
    from fem_b200 import fields
    d = _need("c2_128")
    rho = fields.smooth_cell(128, 4.0, seed=2)
    assert rho.sum() == pytest.approx(d["rho_sum"], rel=1e-12)
    ref = np.array(d["C"]).reshape(6, 6)
    for prec, tol in _modes(femh):
        C, info = femh.Engine(precision=prec).homogenize(rho)
        assert info["status"] == 0 and _rel(C, ref) < tol, (prec, _rel(C, ref))


def test_c3_256_binary_cell(femh):
    """C3 in every precision mode: plain FP64, FP64 CG with the FP32 V-cycle,
    and FP32 inner PCG in FP64 defect correction.  (BF16 storage of the
    search directions does not converge on this cell: measured, see the
    store_bf16 option.)"""
    from fem_b200 import fields
    d = _need("c3_256")
    rho = fields.median_cell(256, 8.0, seed=3)
    assert rho.sum() == pytest.approx(d["rho_sum"], rel=1e-12)
    ref = np.array(d["C"]).reshape(6, 6)
    cases = [(dict(precision=femh.FP64), TOL_FP64), (dict(precision=femh.MIXED_PC), TOL_MIXED),
             (dict(precision=femh.MIXED, inner_tol=1e-3, max_outer=10), TOL_MIXED)]
    for kw, tol in cases:
        e = femh.Engine(**kw)
        C, info = e.homogenize(rho)
        assert info["status"] == 0 and _rel(C, ref) < tol, (kw, _rel(C, ref))
        e.close()


@pytest.mark.parametrize("n", [64, 128])
def test_c4_gradient(femh, n):
    from fem_b200 import fields
    d = _need(f"c4_{n}")
    rho = fields.smooth_cell(n, 4.0, seed=4)
    assert rho.sum() == pytest.approx(d["rho_sum"], rel=1e-12)
    Ct = np.array(d["C_target"]).reshape(6, 6)
    ref = np.array(d["C"]).reshape(6, 6)
    vox = np.array(d["voxels"])
    gref = np.array(d["dLdrho"])
    for prec, tol in _modes(femh):
        e = femh.Engine(precision=prec)
        C, info = e.homogenize(rho)
        assert info["status"] == 0 and _rel(C, ref) < tol
        g = e.grad(2.0 * (C - Ct)).ravel()
        assert _rel(g[vox], gref) < TOL_GRAD, (prec, _rel(g[vox], gref))
        assert g.sum() == pytest.approx(d["dLdrho_sum"], rel=TOL_GRAD, abs=TOL_GRAD * np.abs(gref).max())
        assert (g * g).sum() == pytest.approx(d["dLdrho_sumsq"], rel=TOL_GRAD)
        e.close()


def test_c5_subset_batched(femh):
    from fem_b200 import fields
    d = _need("c5_64")
    cells = fields.uneven_batch(4096, seed=7, count=len(d["cells"]))
    for c, rec in zip(cells, d["cells"]):
        assert c.shape[0] == rec["n"] and c.sum() == rec["rho_sum"]
    ref = np.array([rec["C"] for rec in d["cells"]]).reshape(-1, 6, 6)
    assert any(c.shape[0] == 64 for c in cells) and any(c.shape[0] == 48 for c in cells)
    for prec, tol in _modes(femh):
        e = femh.Engine(precision=prec)
        C, infos, _ = e.batch(cells)
        assert all(i["status"] == 0 for i in infos)
        errs = [_rel(C[k], ref[k]) for k in range(len(cells))]
        assert max(errs) < tol, (prec, max(errs), int(np.argmax(errs)))
        e.close()
