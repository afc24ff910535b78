"""Size-independent properties at full workload sizes, where the oracle would
take minutes (all through the C ABI):
  * the operator at 128^3: symmetry u.Kv = v.Ku, linearity, rigid
    translations in its null space (FP64), and the packed-FP32x2 kernels
    against the FP64 operator (2e-6 relative, max-norm);
  * C^H of the 128^3 smooth-field workload: mixed precision (FP64 CG, FP32
    multigrid) against plain FP64 within the mixed bar 1e-6, symmetric and
    positive definite;
  * C^H at 64^3 under an axis swap (x<->y permutes the Voigt entries) and a
    periodic translation of the cell (unchanged), within the FP64 bar 1e-8.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-8
TOL_MIXED = 1e-6
TOL_APPLY32 = 2e-6


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.fixture(scope="module")
def cell128():
    from fem_b200 import fields
    return fields.smooth_cell(128, 4.0, seed=2)


def test_operator_properties_128(femh, cell128):
    rng = np.random.default_rng(3)
    shape = (6,) + cell128.shape + (3,)
    u = rng.standard_normal(shape)
    v = rng.standard_normal(shape)
    e = femh.Engine()
    Ku = e.apply_operator(cell128, u)
    Kv = e.apply_operator(cell128, v)
    for I in range(6):
        a = np.vdot(v[I], Ku[I])
        b = np.vdot(u[I], Kv[I])
        scale = np.sqrt(np.vdot(Ku[I], Ku[I]) * np.vdot(v[I], v[I]))
        assert abs(a - b) <= 1e-12 * scale
    Kw = e.apply_operator(cell128, 2.0 * u - 0.5 * v)
    assert _rel(Kw, 2.0 * Ku - 0.5 * Kv) < 1e-13
    t = np.broadcast_to(np.array([1.0, -2.0, 0.5]), shape).copy()
    Kt = e.apply_operator(cell128, t)
    assert np.abs(Kt).max() <= 1e-12 * np.abs(Ku).max()


@pytest.mark.parametrize("variant", [3, 4, 5, 7])
def test_fp32_packed_kernels_128(femh, cell128, variant):
    rng = np.random.default_rng(4)
    u = rng.standard_normal((6,) + cell128.shape + (3,))
    y64 = femh.Engine().apply_operator(cell128, u)
    y32 = femh.Engine(precision=femh.MIXED_PC, stencil_variant=variant, autotune=0).apply_operator(cell128, u)
    assert _rel(y32, y64) < TOL_APPLY32


def test_mixed_pc_vs_fp64_128(femh, cell128):
    C64, i64 = femh.Engine().homogenize(cell128)
    Cm, im = femh.Engine(precision=femh.MIXED_PC).homogenize(cell128)
    assert i64["status"] == 0 and im["status"] == 0
    assert max(im["rel_residual"]) < 1e-10
    assert _rel(Cm, C64) < TOL_MIXED
    assert np.abs(Cm - Cm.T).max() <= 1e-12 * np.abs(Cm).max()
    assert np.linalg.eigvalsh(0.5 * (Cm + Cm.T)).min() > 0


def test_axis_swap_and_translation_64(femh):
    from fem_b200 import fields
    rho = fields.smooth_cell(64, 4.0, seed=7)
    e = femh.Engine()
    C, _ = e.homogenize(rho)
    Cs, _ = e.homogenize(np.ascontiguousarray(rho.transpose(1, 0, 2)))
    perm = [1, 0, 2, 4, 3, 5]   # xx<->yy, yz<->xz
    assert _rel(Cs, C[np.ix_(perm, perm)]) < TOL_FP64
    Ct, _ = e.homogenize(np.ascontiguousarray(np.roll(rho, (5, 7, 11), axis=(0, 1, 2))))
    assert _rel(Ct, C) < TOL_FP64


def test_persistent_staged_kernel_same_bits_128(femh, cell128):
    """The staged FP32 kernel as persistent CTAs (variant 7: one CTA per
    multiprocessor and load case group, each streaming a balanced run of
    units) against one CTA per unit (variant 5) on the same units: the
    operator, and a whole mixed-precision solve whose V-cycles run the Jacobi,
    residual and Jacobi+dot sweeps, give the same bits."""
    rng = np.random.default_rng(6)
    u = rng.standard_normal((6,) + cell128.shape + (3,))
    e5 = femh.Engine(precision=femh.MIXED_PC, stencil_variant=5, autotune=0)
    e7 = femh.Engine(precision=femh.MIXED_PC, stencil_variant=7, autotune=0)
    assert np.array_equal(e5.apply_operator(cell128, u), e7.apply_operator(cell128, u))
    C5, i5 = e5.homogenize(cell128)
    C7, i7 = e7.homogenize(cell128)
    assert i5["status"] == 0 and i7["status"] == 0
    assert i5["iterations"] == i7["iterations"]
    assert np.array_equal(C5, C7)


def test_persistent_staged_kernel_batch(femh):
    """Persistent CTAs whose runs span several cells of a batch, with the unit
    lists compacted (and the CTA tables rebuilt) as cells converge: C^H and
    iterations of every cell are the same bits as with one CTA per unit."""
    from fem_b200 import fields
    rhos = [fields.binary_cell(32, vf, seed=s) for s, vf in ((1, 0.25), (2, 0.5), (3, 0.35), (4, 0.6), (5, 0.45))]
    rhos.append(fields.smooth_cell(32, 3.0, seed=9))
    out = {}
    for var in (5, 7):
        C, infos, _ = femh.Engine(precision=femh.MIXED_PC, stencil_variant=var, autotune=0).batch(rhos, h=None)
        out[var] = (C, [i["iterations"] for i in infos], [i["status"] for i in infos])
    assert out[5][2] == [0] * len(rhos) and out[7][2] == [0] * len(rhos)
    assert out[5][1] == out[7][1]
    assert np.array_equal(out[5][0], out[7][0])
