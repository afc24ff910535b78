"""The oracle's multigrid PCG (oracle/femh_oracle_mg.c) against its plain
Jacobi-PCG restatement (oracle/femh_oracle.c) and closed forms, on the CPU:

* the Hadamard-form operator apply equals the dense element-by-element apply
  (odd extents, z extents that are not multiples of the vector block);
* C^H of random binary and smooth cells, cubic and not, agrees with the
  Jacobi-PCG solve to 1e-12 relative; the uniform cell gives the isotropic C;
* the multigrid fluctuation equals the Jacobi one (the same periodic problem).
"""
import numpy as np
import pytest


@pytest.mark.parametrize("shape", [(2, 2, 2), (4, 4, 4), (5, 3, 7), (6, 4, 8), (3, 5, 70), (2, 2, 130)])
def test_mg_apply_equals_dense_apply(oracle, shape):
    rng = np.random.default_rng(sum(shape))
    c = rng.uniform(0.1, 1.0, shape)
    u = rng.standard_normal((6,) + shape + (3,))
    y = oracle.apply(shape, oracle.k0(1.0, 0.3, 1.0), c.ravel(), u)
    y[:, 0, 0, 0, :] = 0.0   # the multigrid operator pins node 0
    ym = oracle.mg_apply(shape, c, u)
    assert np.abs(ym - y).max() < 1e-14 * np.abs(y).max()


@pytest.mark.parametrize("shape,kind", [((8, 8, 8), "binary"), ((8, 12, 16), "binary"),
                                        ((12, 12, 12), "smooth"), ((6, 6, 6), "binary")])
def test_mg_homogenize_matches_jacobi(oracle, shape, kind):
    rng = np.random.default_rng(shape[0] * 7 + shape[2])
    rho = (rng.random(shape) < 0.5).astype(float) if kind == "binary" else 1e-3 + rng.random(shape)
    C, chi, it, rel, st = oracle.homogenize(rho, tol=1e-12, max_iter=100000)
    Cm, chim, itm, relm, stm = oracle.mg_homogenize(rho, tol=1e-12)
    assert st == 0 and stm == 0
    assert max(relm) < 1e-12
    assert max(itm) < max(it) / 4   # the point of the multigrid preconditioner
    assert np.abs(Cm - C).max() < 1e-12 * np.abs(C).max()
    assert np.abs(chim - chi).max() < 1e-9 * np.abs(chi).max()


def test_mg_uniform_cell_is_isotropic(oracle):
    rho = np.ones((8, 8, 8))
    C, _, it, _, st = oracle.mg_homogenize(rho, tol=1e-12)
    assert st == 0
    assert np.abs(C - oracle.c_iso(1.0, 0.3)).max() < 1e-12


def test_mg_jacobi_smoother_setting(oracle):
    """cheb_ratio 0 (every sweep damped by 0.35) and 2 + 2 sweeps still converge
    to the same C^H."""
    rng = np.random.default_rng(11)
    rho = (rng.random((8, 8, 8)) < 0.5).astype(float)
    C = oracle.mg_homogenize(rho, tol=1e-12)[0]
    C2, _, it2, _, st2 = oracle.mg_homogenize(rho, tol=1e-12, pre=2, post=2, cheb_ratio=0.0)
    assert st2 == 0
    assert np.abs(C2 - C).max() < 1e-12 * np.abs(C).max()


@pytest.mark.parametrize("shape,kind", [((8, 8, 8), "binary"), ((8, 12, 16), "binary"), ((12, 12, 12), "smooth")])
def test_mg_block_smoother(oracle, shape, kind):
    """The node-block Jacobi sweeps (the 3x3 diagonal block of K inverted at
    every node, the Chebyshev interval from the block-scaled element bound)
    solve the same problem: C^H equals the point-Jacobi multigrid's to 1e-12,
    in no more iterations on these contrast-1e6 cells."""
    rng = np.random.default_rng(shape[1] * 5 + shape[2])
    rho = (rng.random(shape) < 0.4).astype(float) if kind == "binary" else 1e-3 + rng.random(shape)
    Cp, _, itp, _, stp = oracle.mg_homogenize(rho, tol=1e-12, want_chi=False)
    Cb, _, itb, relb, stb = oracle.mg_homogenize(rho, tol=1e-12, want_chi=False, block=True)
    assert stp == 0 and stb == 0
    assert max(relb) < 1e-12
    assert np.abs(Cb - Cp).max() < 1e-12 * np.abs(Cp).max()
    assert max(itb) <= max(itp)
