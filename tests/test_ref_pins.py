"""Restatements pinned to the reference's OWN code, run on the CPU.

oracle/build_ref.sh compiles the reference's sources in place into
oracle/_ref/ (tests skip without the reference tree at build time):

* SamplesGenerator's NumericalCoarsening (force-driven coarsened tensor and
  parameters, SamplesGenerator/NumericalCoarsening.cpp:266-340) as shipped
  (float, 1 + 1e-5 diagonal scaling), with Eigen's sparse LU in place of the
  absent PARDISO, against oracle/femlib_force.py (regularised): cubic and
  general structure types, cubic and non-cubic cells.  Tolerance 2e-5 relative
  (the reference computes in float).
"""
import numpy as np
import pytest

from oracle import femlib_force as FF
from oracle import ref as R

pytestmark = pytest.mark.skipif(not R.available("libnc_ref.so"), reason="oracle/_ref/libnc_ref.so not built")

TOL_FLOAT = 2e-5


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


@pytest.mark.parametrize("shape,seed", [((2, 2, 2), 1), ((3, 3, 3), 2), ((4, 4, 4), 3), ((5, 5, 5), 4)])
def test_nc_cubic_reference_vs_restatement(shape, seed):
    mats = (np.random.default_rng(seed).random(shape) < 0.5).astype(np.int32)
    E, nu, dens = (0.1, 1.0), 0.3, (0.0, 1.0)
    tv, pv = R.nc_coarsen(mats, E, nu, dens, R.CUBIC)
    _, tv2, pv2 = FF.coarsen(mats.ravel(), shape, np.array(E), nu, dens=dens, cubic=True, regularize=True)
    assert _rel(tv, tv2) < TOL_FLOAT
    assert pv.size == 4 and _rel(pv, pv2) < TOL_FLOAT


@pytest.mark.parametrize("shape,seed", [((4, 4, 4), 5), ((2, 3, 4), 6), ((4, 6, 8), 7)])
def test_nc_general_reference_vs_restatement(shape, seed):
    """General structure type (three Y, three nu, three G) -- on non-cubic cells
    as well, where femlib's shear loads are out of moment balance: the
    restatement follows the reference there too."""
    mats = (np.random.default_rng(seed).random(shape) < 0.6).astype(np.int32)
    E, nu, dens = (0.2, 1.0), 0.3, (0.0, 1.0)
    tv, pv = R.nc_coarsen(mats, E, nu, dens, R.GENERAL)
    _, tv2, pv2 = FF.coarsen(mats.ravel(), shape, np.array(E), nu, dens=dens, cubic=False, regularize=True)
    assert _rel(tv, tv2) < TOL_FLOAT
    assert pv.size == 10 and _rel(pv, pv2) < TOL_FLOAT


def test_nc_uniform_reference_is_material():
    """A uniform cell under the reference's own code returns the material's
    Y, nu and G within the 1e-5 diagonal scaling."""
    mats = np.ones((3, 3, 3), np.int32)
    tv, pv = R.nc_coarsen(mats, (0.5, 1.0), 0.3, (0.0, 1.0), R.CUBIC)
    mu = 1.0 / (2 * 1.3)
    assert np.allclose(pv, [1.0, 1.0, 0.3, mu], rtol=1e-4, atol=0)


# ---------------------------------------------------------------- fast_fem FEM3DFun
def _ff_case(n, m, seed):
    rng = np.random.default_rng(seed)
    x0 = rng.uniform(-0.1, 1.1, m ** 3)   # outside [1e-3, 1] too: setParam clamps
    G0 = np.diag([0.1, 0.1, 0.1, 0.03, 0.03, 0.03]) + 0.01 * np.triu(np.ones((6, 6)), 1)
    wG = np.triu(rng.uniform(0.5, 1.5, (6, 6)))
    return x0, G0, wG


@pytest.mark.skipif(not R.available("libfastfem_ref.so"), reason="oracle/_ref/libfastfem_ref.so not built")
@pytest.mark.parametrize("n,m", [(8, 8), (8, 4), (12, 6)])
def test_fastfem_energy_and_gradient_loops_vs_oracle(oracle, n, m):
    """fast_fem's own setParam energy loop, f and df (field chain rule and
    density term included, fast_fem/FEM3DFun.cpp:128-268), fed the oracle's
    fluctuation through the stand-in topoOptLib headers, against the oracle's
    energy and gradient restatement (fo_energy, fo_grad) on the same clamped
    distribution: G to 1e-12, df to 1e-10 relative.  The reference fills only
    the upper triangle of G; with upper-triangular weights its objective is the
    symmetric one."""
    x0, G0, wG = _ff_case(n, m, seed=n + m)
    nu, m0, mw = 0.3, 0.4, 0.1
    r = R.fastfem(n, x0, nu, G0, wG, m0, mw)
    assert r["status"] == 0
    rep = n // m
    rho = np.clip(np.repeat(np.repeat(np.repeat(x0.reshape(m, m, m), rep, 0), rep, 1), rep, 2), 1e-3, 1.0)
    assert np.array_equal(r["distribution"], rho)
    assert r["density"] == pytest.approx(rho.mean(), rel=1e-14)
    mat = oracle.material(interp=oracle.INTERP_RAMP3, E_s=1.0, nu=nu)
    C, chi, _, _, st = oracle.homogenize(rho, mat=mat, tol=1e-12, max_iter=100000)
    assert st == 0
    iu = np.triu_indices(6)
    assert np.abs(r["G"][iu] - C[iu]).max() < 1e-11 * np.abs(C).max()
    assert np.abs(np.tril(r["G"], -1)).max() == 0.0
    Gref = r["G"]
    f = 0.5 * np.sum(wG * (Gref - G0) ** 2) + 0.5 * mw * (rho.mean() - m0) ** 2
    assert r["f"] == pytest.approx(f, rel=1e-10)
    dfd = oracle.grad(rho, chi, wG * (Gref - G0), mat=mat) + (mw / rho.size) * (rho.mean() - m0)
    g = dfd.reshape(m, rep, m, rep, m, rep).sum(axis=(1, 3, 5)).ravel()
    assert np.abs(r["df"] - g).max() < 1e-10 * np.abs(g).max()



@pytest.mark.skipif(not R.available("libfastfem_ref.so"), reason="oracle/_ref/libfastfem_ref.so not built")
@pytest.mark.parametrize("kind", [R.FIELD_SYM, R.FIELD_CUBIC])
def test_fastfem_symmetric_fields_vs_oracle(oracle, kind):
    """The same loops over the mirror- and cubic-symmetric fields of
    fast_fem/PiecewiseConstant{Sym,Cubic}3D.cpp (the cubic one is run3D's,
    fast_fem/run3d.cpp:176-182): the chain rule sums every voxel into the
    parameter the field assigns it."""
    n, m = 8, 4
    x0, G0, wG = _ff_case(n, m, seed=30 + kind)
    nu, m0, mw = 0.3, 0.4, 0.1
    r = R.fastfem(n, x0, nu, G0, wG, m0, mw, kind=kind)
    assert r["status"] == 0
    idx = np.array([R.field_index(kind, m, ((i + .5) / n, (j + .5) / n, (k + .5) / n))
                    for i in range(n) for j in range(n) for k in range(n)])
    rho = np.clip(x0[idx], 1e-3, 1.0).reshape(n, n, n)
    assert np.array_equal(r["distribution"], rho)
    mat = oracle.material(interp=oracle.INTERP_RAMP3, E_s=1.0, nu=nu)
    C, chi, _, _, st = oracle.homogenize(rho, mat=mat, tol=1e-12, max_iter=100000)
    iu = np.triu_indices(6)
    assert np.abs(r["G"][iu] - C[iu]).max() < 1e-11 * np.abs(C).max()
    dfd = oracle.grad(rho, chi, wG * (r["G"] - G0), mat=mat) + (mw / rho.size) * (rho.mean() - m0)
    g = np.bincount(idx, weights=dfd.ravel(), minlength=m ** 3)
    assert np.abs(r["df"] - g).max() < 1e-10 * np.abs(g).max()
