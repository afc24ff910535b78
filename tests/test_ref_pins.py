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
