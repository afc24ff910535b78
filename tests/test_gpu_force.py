"""femh_force_tensors (femlib's force-driven coarse tensor, evaluated on the
engine's strain-driven fields) against the oracle's restatement of femlib's
multiplier system (oracle/femlib_force.py), through the C ABI.

Bars: FP64 solve 1e-8 relative (max entry / max |C|), mixed precision 1e-6,
as for C^H.  The oracle runs without femlib's 1e-5 diagonal scaling (the
engine computes the exact value; test_oracle.py bounds that scaling's effect
by 1e-4).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E2, NU2 = (0.26, 1.0), 0.3
TOL = {"fp64": 1e-8, "mixed_pc": 1e-6}


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _cell(n, seed):
    return (np.random.default_rng(seed).random((n, n, n)) < 0.5).astype(int)


def _engine(femh, precision):
    prec = {"fp64": femh.FP64, "mixed_pc": femh.MIXED_PC}[precision]
    return femh.Engine(precision=prec, interp=2, bin_hi=E2[1], bin_lo=E2[0], nu=NU2)


@pytest.mark.parametrize("precision", ["fp64", "mixed_pc"])
@pytest.mark.parametrize("n", [4, 6, 8])
def test_force_tensor_matches_femlib_restatement(femh, n, precision):
    from oracle import femlib_force as ff
    mats = _cell(n, seed=n)
    Cref, _, _ = ff.coarsen(mats.ravel(), (n, n, n), E2, NU2, regularize=False)
    e = _engine(femh, precision)
    C, info = e.homogenize(mats.astype(float), h=1.0 / n)
    assert info["status"] == 0
    Cf = e.force_tensors()
    assert _rel(Cf, Cref) < TOL[precision]
    assert np.abs(Cf - Cf.T).max() <= 1e-12 * np.abs(Cf).max()
    assert _rel(Cf, C) > 1e-3   # femlib's shear convention: not C^H for a non-uniform cell


def test_force_tensor_of_uniform_cell_is_the_material(femh):
    from oracle import femlib_force as ff
    e = _engine(femh, "fp64")
    e.homogenize(np.ones((8, 8, 8)), h=1.0 / 8)
    assert _rel(e.force_tensors(), ff.iso_matrix(E2[1], NU2)) < 1e-12


def test_force_tensors_of_a_batch(femh):
    """One batched solve of cubic cells of three sizes: each cell's tensor."""
    from oracle import femlib_force as ff
    cells = [_cell(n, seed=10 + n) for n in (4, 6, 8)]
    e = _engine(femh, "fp64")
    e.batch([c.astype(float) for c in cells])
    Cf = e.force_tensors()
    assert Cf.shape == (3, 6, 6)
    for c, got in zip(cells, Cf):
        n = c.shape[0]
        ref, _, _ = ff.coarsen(c.ravel(), (n, n, n), E2, NU2, regularize=False)
        assert _rel(got, ref) < TOL["fp64"]


def test_force_tensor_rejects_noncubic_cells(femh):
    e = _engine(femh, "fp64")
    e.homogenize(np.ones((4, 6, 8)), h=1.0 / 8)
    with pytest.raises(femh.FemhError) as ex:
        e.force_tensors()
    assert ex.value.code == 1   # FEMH_E_ARG


def test_force_tensor_before_a_solve_is_a_state_error(femh):
    e = _engine(femh, "fp64")
    with pytest.raises(femh.FemhError):
        e.force_tensors()
