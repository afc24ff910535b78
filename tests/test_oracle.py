"""CPU checks of the FP64 oracle against the reference's golden fixture and
closed-form known answers (pins the oracle before it is trusted as the
checker of the GPU engine)."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "k0_lkh8_nu045.txt")
# lk_H8 node a <-> z-fastest `oneV` node (fast_fem/FEM3DFun.cpp:58-60)
LKH8_TO_ONEV = [0, 4, 6, 2, 1, 5, 7, 3]


def _golden_k0():
    return np.loadtxt(GOLDEN, comments="#")


def test_k0_matches_reference_fixture(oracle):
    """K0(E=1, nu=0.45, h=1) equals the reference's tests/1.K (lk_H8 order)."""
    K = oracle.k0(1.0, 0.45, 1.0)
    idx = [3 * LKH8_TO_ONEV[a] + c for a in range(8) for c in range(3)]
    ref = _golden_k0()
    assert np.abs(K[np.ix_(idx, idx)] - ref).max() < 1e-12


def test_k0_properties(oracle):
    for nu in (0.0, 0.3, 0.45):
        K = oracle.k0(2.0, nu, 0.25)
        assert np.abs(K - K.T).max() < 1e-14
        # rigid translations are in the null space
        for c in range(3):
            t = np.zeros(24)
            t[c::3] = 1
            assert np.abs(K @ t).max() < 1e-13
        w = np.linalg.eigvalsh(K)
        assert (w > -1e-12).all() and (w > 1e-10).sum() == 18
        # K0 scales with E * h in 3-D
        assert np.allclose(oracle.k0(1.0, nu, 1.0) * 2.0 * 0.25, K, atol=1e-14)


def test_uniform_cell_is_isotropic(oracle):
    rho = np.ones((6, 6, 6))
    C, chi, it, rel, st = oracle.homogenize(rho)
    assert st == 0
    assert np.abs(C - oracle.c_iso(1.0, 0.3)).max() < 1e-12


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_voxel_laminate_exact(oracle, axis):
    """A layered cell's FE solution is piecewise linear across the layers and
    is represented exactly by trilinear voxels: C^H = laminate formula."""
    n = 8
    prof = np.array([1.0, 0.3, 0.3, 1.0, 0.6, 0.2, 1.0, 0.9])
    shape = [1, 1, 1]
    shape[axis] = n
    rho = np.broadcast_to(prof.reshape(shape), (n, n, n)).copy()
    mat = oracle.material()
    C, chi, it, rel, st = oracle.homogenize(rho, mat=mat)
    Es = [oracle.lib().fo_coef(mat, float(r)) for r in prof]
    Cref = oracle.c_laminate(Es, 0.3, axis)
    assert np.abs(C - Cref).max() < 1e-9 * np.abs(Cref).max()


def test_axis_permutation_equivariance(oracle):
    rng = np.random.default_rng(3)
    rho = (rng.random((6, 6, 6)) < 0.6).astype(float)
    C, *_ = oracle.homogenize(rho)
    # swap x and y: Voigt xx<->yy, yz<->xz
    P = [1, 0, 2, 4, 3, 5]
    C2, *_ = oracle.homogenize(np.ascontiguousarray(rho.transpose(1, 0, 2)))
    assert np.abs(C2 - C[np.ix_(P, P)]).max() < 1e-8 * np.abs(C).max()
    # periodic translation invariance
    C3, *_ = oracle.homogenize(np.roll(rho, (2, 1, 3), axis=(0, 1, 2)))
    assert np.abs(C3 - C).max() < 1e-8 * np.abs(C).max()


def test_energy_gradient_vs_finite_differences(oracle):
    """dL/drho of L = ||C - Ct||_F^2 from the adjoint formula against central
    differences of the full solve (the reference's check_df pattern,
    fast_fem/run3d.cpp:291-323)."""
    rng = np.random.default_rng(4)
    n = 4
    rho = 0.3 + 0.6 * rng.random((n, n, n))
    mat = oracle.material()
    C, chi, *_ = oracle.homogenize(rho, mat=mat, tol=1e-13)
    Ct = oracle.c_iso(0.2, 0.3)
    dLdC = 2 * (C - Ct)
    g = oracle.grad(rho, chi, dLdC, mat=mat)
    hstep = 1e-6
    for flat in rng.choice(n ** 3, 5, replace=False):
        i = np.unravel_index(flat, rho.shape)
        rp = rho.copy(); rp[i] += hstep
        rm = rho.copy(); rm[i] -= hstep
        Lp = np.sum((oracle.homogenize(rp, mat=mat, tol=1e-13)[0] - Ct) ** 2)
        Lm = np.sum((oracle.homogenize(rm, mat=mat, tol=1e-13)[0] - Ct) ** 2)
        fd = (Lp - Lm) / (2 * hstep)
        assert abs(fd - g[i]) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(g).max())


def test_dCdrho_consistent_with_grad(oracle):
    rng = np.random.default_rng(5)
    rho = 0.2 + 0.7 * rng.random((4, 4, 4))
    C, chi, *_ = oracle.homogenize(rho)
    d = oracle.dCdrho(rho, chi)
    W = rng.standard_normal((6, 6))
    g = oracle.grad(rho, chi, W)
    t = 0
    acc = np.zeros_like(rho)
    for I in range(6):
        for J in range(I + 1):
            acc += d[t] * (W[I, I] if I == J else W[I, J] + W[J, I])
            t += 1
    assert np.abs(acc - g).max() < 1e-12 * np.abs(g).max()


def test_k0_matches_reference_femlib_code(oracle):
    """The reference's own femlib element code (compiled from its sources by
    oracle/build_ref.sh, FP64) gives the same K0 up to its float Gauss points
    (femlib/src/Quadrature.cpp:3-7): ~1e-8."""
    import ctypes
    path = os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref", "libfemlib_ref.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    L = ctypes.CDLL(path)
    for nu in (0.3, 0.45):
        K = np.zeros((24, 24))
        assert L.femlib_k0(ctypes.c_double(1.0), ctypes.c_double(nu), K.ctypes.data_as(ctypes.c_void_p)) == 0
        assert np.abs(K - oracle.k0(1.0, nu, 1.0)).max() < 2e-8


# ---------------------------------------------------------------- femlib's force-driven coarsening
E2, NU2 = (0.26, 1.0), 0.3


def _binary(n, seed):
    return (np.random.default_rng(seed).random(n) < 0.5).astype(int).ravel()


def test_femlib_force_homogeneous_is_isotropic():
    """Face-force loading of a uniform cubic cell returns the material itself:
    C = E(nu), Y = E, nu_xy = nu, G = mu (without the 1e-5 diagonal scaling
    exactly; with it within that scaling)."""
    from oracle import femlib_force as ff
    mats = np.ones(27, int)
    iso = ff.iso_matrix(1.0, NU2)
    for reg, tol in ((False, 1e-12), (True, 1e-4)):
        C, tv, pv = ff.coarsen(mats, (3, 3, 3), E2, NU2, regularize=reg)
        assert np.abs(C - iso).max() < tol
        assert np.allclose(pv, [1.0, 1.0, NU2, iso[3, 3]], rtol=tol, atol=0)
        assert tv.size == 21


@pytest.mark.parametrize("n", [4, 5])
def test_femlib_force_tensor_equals_strain_driven_route(n):
    """On a cubic binary cell femlib's multiplier system (face forces, periodic
    jumps, fixed mean translation and rotation) gives the same tensor as S W' S
    evaluated on the six strain-driven fluctuation fields -- the route the
    engine takes -- and its coarse strains are (C^H)^-1 sigma, so Y and nu
    follow from the compliance."""
    from oracle import femlib_force as ff, oracle as O
    mats = _binary((n, n, n), seed=n)
    us, X, nn = ff.harmonic_displacements(mats, (n, n, n), E2, NU2, regularize=False)
    C = ff.femlib_tensor(us, X, nn, mats, E2, NU2)
    Cf = ff.tensor_from_fields(mats, (n, n, n), E2, NU2)
    assert np.abs(C - Cf).max() < 1e-10 * np.abs(Cf).max()
    assert np.abs(C - C.T).max() < 1e-12 * np.abs(C).max()
    rho = (mats.reshape(n, n, n) == 1).astype(float)
    mat = O.material(interp=O.INTERP_BINARY, nu=NU2, bin_hi=E2[1], bin_lo=E2[0])
    CH = O.homogenize(rho, h=1.0 / n, mat=mat, tol=1e-13, max_iter=200000)[0]
    S = np.linalg.inv(CH)
    for a in range(3):   # unit stress on the unit cube's faces
        eps = ff._voigt_t(ff.coarse_strain(us[a], X, nn))
        assert np.abs(eps[:3] - S[:3, a]).max() < 1e-10 * abs(S[a, a])
    # femlib's shear convention makes C differ from C^H once the cell is not uniform
    assert np.abs(C - CH).max() > 1e-3 * np.abs(CH).max()
    # the 1e-5 diagonal scaling moves the tensor by about that much
    Cr = ff.femlib_tensor(*ff.harmonic_displacements(mats, (n, n, n), E2, NU2, regularize=True), mats, E2, NU2)
    assert np.abs(Cr - C).max() < 1e-4 * np.abs(C).max()


def test_femlib_force_noncubic_shear_loads_unbalanced():
    """Why the engine's force-driven tensor is defined for cubic cells only: on
    a uniform 4x6x8 cell femlib's shear face loads (f/2 on faces of different
    areas) are out of moment balance, the rotation multipliers load the
    interior, and the tensor is no longer the material's."""
    from oracle import femlib_force as ff
    n = (4, 6, 8)
    C, _, _ = ff.coarsen(np.ones(4 * 6 * 8, int), n, E2, NU2, regularize=False)
    assert np.abs(C - ff.iso_matrix(1.0, NU2)).max() > 1e-3
