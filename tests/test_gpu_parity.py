"""GPU parity of the CUDA engine (through the C ABI) against the FP64 oracle.

Bars (the accuracy required of this path: C^H 1e-8 FP64 / 1e-6 mixed, gradients 1e-5):
  * operator apply, FP64:                 1e-13 relative (max-norm)
  * operator apply, FP32 kernels:         2e-6 relative (max-norm; FP32 rounding
                                          of rho-scaled coefficients, u and sums)
  * C^H, plain FP64 (Jacobi / GMG PCG):   1e-8 relative (max entry / max |C|)
  * C^H, mixed precision (FP32 inner):    1e-6 relative
  * gradients dL/drho, dC/drho:           1e-5 relative
Sizes are the ones the oracle finishes in seconds; full-size cases are covered
by size-independent properties in test_gpu_properties.py.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_APPLY = 1e-13
TOL_APPLY32 = 2e-6
TOL_FP64 = 1e-8
TOL_MIXED = 1e-6
TOL_GRAD = 1e-5


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.fixture(scope="module")
def rng():
    return np.random.default_rng(11)


@pytest.mark.parametrize("shape", [(8, 8, 8), (6, 10, 4), (16, 16, 16), (12, 8, 20)])
def test_apply_matches_oracle(femh, oracle, rng, shape):
    rho = rng.random(shape)
    u = rng.standard_normal((6,) + shape + (3,))
    e = femh.Engine()
    y = e.apply_operator(rho, u)
    mat = oracle.material()
    yo = oracle.apply(shape, oracle.k0(1.0, 0.3, 1.0 / shape[0]), oracle.coef(mat, rho), u)
    assert _rel(y, yo) < TOL_APPLY


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 7])
@pytest.mark.parametrize("shape", [(16, 16, 16), (12, 8, 20), (8, 24, 24), (6, 10, 4), (8, 16, 128),
                                   (6, 20, 64), (4, 32, 32), (5, 11, 128), (3, 5, 16), (4, 6, 256)])
def test_fp32_stencil_variants_match_oracle(femh, oracle, rng, shape, variant):
    """The FP32 kernels of the multigrid sweeps, each forced in turn: one voxel
    row per thread, two rows per thread, two load cases per thread in packed
    FP32x2 lanes, two rows per thread in packed FP32x2 lanes, the same with
    its inputs staged by bulk copies, and that one as persistent CTAs.  z extents in the compile-time set run
    the compile-time kernels (the staged one up to 128; at 256 it falls back
    to the unstaged packed kernel), the others (20, 4) the runtime-z kernels;
    in (3, 5, 16) and (16, 16, 16) one tile covers the whole y ring, so the
    staged rows wrap around it."""
    rho = 0.3 + 0.7 * rng.random(shape)
    u = rng.standard_normal((6,) + shape + (3,))
    e = femh.Engine(precision=femh.MIXED_PC, solver=femh.JACOBI_PCG, stencil_variant=variant, autotune=0)
    y = e.apply_operator(rho, u)
    mat = oracle.material()
    yo = oracle.apply(shape, oracle.k0(1.0, 0.3, 1.0 / shape[0]), oracle.coef(mat, rho), u)
    assert _rel(y, yo) < TOL_APPLY32


@pytest.mark.parametrize("shape", [(8, 16, 128), (6, 20, 64), (4, 32, 32), (5, 11, 128), (3, 5, 16), (4, 6, 256)])
def test_fp64_staged_apply_matches_oracle(femh, oracle, rng, shape):
    """The FP64 kernel with bulk-copy staged inputs (forced; these shapes meet
    its row condition) against the oracle operator at the FP64 bar."""
    rho = rng.random(shape)
    u = rng.standard_normal((6,) + shape + (3,))
    e = femh.Engine(solver=femh.JACOBI_PCG, stencil_variant=6, autotune=0)
    y = e.apply_operator(rho, u)
    mat = oracle.material()
    yo = oracle.apply(shape, oracle.k0(1.0, 0.3, 1.0 / shape[0]), oracle.coef(mat, rho), u)
    assert _rel(y, yo) < TOL_APPLY


@pytest.mark.parametrize("precision", ["fp64", "mixed_pc"])
def test_staged_kernels_C_matches_oracle(femh, oracle, precision):
    """C^H with the staged kernels forced (FP64 operator: variant 6; the FP32
    multigrid levels fall back where a level does not qualify)."""
    from fem_b200 import fields
    rho = fields.smooth_cell(64, sigma=3.0, seed=12)[:16, :24, :].copy()
    Co, *_ = oracle.homogenize(rho)
    prec = femh.FP64 if precision == "fp64" else femh.MIXED_PC
    e = femh.Engine(precision=prec, stencil_variant=6)
    C, info = e.homogenize(rho)
    assert info["status"] == 0 and max(info["rel_residual"]) < 1e-10
    assert _rel(C, Co) < (TOL_FP64 if precision == "fp64" else TOL_MIXED)


@pytest.mark.parametrize("bf16", [0, 1])
@pytest.mark.parametrize("shape", [(16, 16, 16), (16, 8, 24)])
def test_mixed_pc_C_matches_oracle(femh, oracle, shape, bf16):
    """FP64 CG with the FP32 multigrid preconditioner (the bench's mixed mode)."""
    from fem_b200 import fields
    rho = fields.smooth_cell(16, sigma=2.0, seed=3)[: shape[0], : shape[1], : shape[2]].copy()
    Co, *_ = oracle.homogenize(rho)
    e = femh.Engine(precision=femh.MIXED_PC, store_bf16=bf16)
    C, info = e.homogenize(rho)
    assert info["status"] == 0 and max(info["rel_residual"]) < 1e-10
    assert _rel(C, Co) < TOL_MIXED


@pytest.mark.parametrize("precision", ["fp64", "mixed_pc", "mixed"])
def test_warm_start_matches_cold(femh, precision):
    """A solve that starts from the previous solution of a nearby density
    field (the descent / line-search case) reaches the same C^H as a cold
    solve of that field, in fewer iterations."""
    from fem_b200 import fields
    prec = {"fp64": femh.FP64, "mixed_pc": femh.MIXED_PC, "mixed": femh.MIXED}[precision]
    rho1 = fields.smooth_cell(32, sigma=3.0, seed=21)
    rng = np.random.default_rng(22)
    rho2 = np.clip(rho1 + 0.01 * rng.standard_normal(rho1.shape), 1e-3, 1.0)
    warm = femh.Engine(precision=prec, warm_start=1)
    warm.homogenize(rho1)
    Cw, iw = warm.homogenize(rho2)
    Cc, ic = femh.Engine(precision=prec).homogenize(rho2)
    assert iw["status"] == 0 and max(iw["rel_residual"]) < 1e-10
    assert _rel(Cw, Cc) < (TOL_FP64 if precision == "fp64" else TOL_MIXED)
    assert sum(iw["iterations"]) < sum(ic["iterations"])
    # the gradient uses the warm-started fields
    dLdC = np.eye(6)
    assert _rel(warm.grad(dLdC), _cold_grad(femh, prec, rho2, dLdC)) < TOL_GRAD


def _cold_grad(femh, prec, rho, dLdC):
    e = femh.Engine(precision=prec)
    e.homogenize(rho)
    return e.grad(dLdC)


def test_apply_deterministic(femh, rng):
    rho = rng.random((16, 16, 16))
    u = rng.standard_normal((6, 16, 16, 16, 3))
    e = femh.Engine()
    assert np.array_equal(e.apply_operator(rho, u), e.apply_operator(rho, u))


@pytest.mark.parametrize("solver", ["jacobi", "gmg"])
@pytest.mark.parametrize("n", [8, 16, 32])
def test_fp64_C_matches_oracle(femh, oracle, n, solver):
    """The 32^3 binary cell (p = 0.5, seed 1) is the CPU parity workload."""
    from fem_b200 import fields
    rho = fields.binary_cell(n, 0.5, seed=1)
    Co, *_ = oracle.homogenize(rho)
    e = femh.Engine(solver=femh.JACOBI_PCG if solver == "jacobi" else femh.GMG_PCG)
    C, info = e.homogenize(rho)
    assert info["status"] == 0 and max(info["rel_residual"]) < 1e-10
    assert _rel(C, Co) < TOL_FP64


@pytest.mark.parametrize("smoothing", [(2, 2, 3.0), (2, 2, 16.0), (3, 3, 16.0), (1, 1, 4.0)])
@pytest.mark.parametrize("precision", ["fp64", "mixed_pc"])
def test_chebyshev_smoother_C_matches_oracle(femh, oracle, precision, smoothing):
    """Chebyshev-root damping weights in the V-cycle (pre sweeps, post sweeps,
    ratio) reach the oracle's C^H on the 32^3 binary cell: the smoother changes
    the iteration count, not the solution."""
    from fem_b200 import fields
    pre, post, ratio = smoothing
    rho = fields.binary_cell(32, 0.5, seed=1)
    Co = _oracle_C(oracle, "binary32", rho)
    prec = {"fp64": femh.FP64, "mixed_pc": femh.MIXED_PC}[precision]
    e = femh.Engine(precision=prec, pre_smooth=pre, post_smooth=post, cheb_ratio=ratio)
    C, info = e.homogenize(rho)
    assert info["status"] == 0 and max(info["rel_residual"]) < 1e-10
    assert _rel(C, Co) < (TOL_FP64 if precision == "fp64" else TOL_MIXED)


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("precision", ["fp64", "mixed_pc"])
def test_block_jacobi_C_matches_oracle(femh, oracle, precision, variant):
    """Node-block Jacobi sweeps (block_jacobi=1: every node's 3x3 diagonal
    block of K inverted, the Chebyshev interval from the block-scaled element
    bound) through each stencil kernel forced in turn (0: the autotuner's
    choice; runtime-z kernels on the coarse levels 12^3 and below) reach the
    oracle's C^H on a 24^3 binary cell, in fewer iterations than point sweeps."""
    from fem_b200 import fields
    rho = fields.binary_cell(24, 0.4, seed=4)
    Co = _oracle_C(oracle, "binary24", rho)
    prec = {"fp64": femh.FP64, "mixed_pc": femh.MIXED_PC}[precision]
    e = femh.Engine(precision=prec, block_jacobi=1, stencil_variant=variant, autotune=1 if variant == 0 else 0)
    C, info = e.homogenize(rho)
    assert info["status"] == 0 and max(info["rel_residual"]) < 1e-10
    assert _rel(C, Co) < (TOL_FP64 if precision == "fp64" else TOL_MIXED)
    if variant == 0:
        _, ip = femh.Engine(precision=prec, block_jacobi=0).homogenize(rho)
        assert max(info["iterations"]) < max(ip["iterations"])


def _block_cell(kind):
    from fem_b200 import fields
    if kind == "smooth24":
        return fields.smooth_cell(24, sigma=1.5, seed=6)
    if kind == "binary24":
        return fields.binary_cell(24, 0.35, seed=8)
    if kind == "laminate16":   # layers along z: some load cases have a zero right-hand side
        prof = np.array([1.0, 0.3, 0.3, 1.0, 0.6, 0.2, 1.0, 0.9] * 2)
        return np.broadcast_to(prof.reshape(1, 1, 16), (16, 16, 16)).copy()
    return np.ascontiguousarray(fields.binary_cell(24, 0.5, seed=9)[:12, :8, :20])


@pytest.mark.parametrize("kind", ["smooth24", "binary24", "laminate16", "noncubic"])
@pytest.mark.parametrize("precision", ["fp64", "mixed_pc", "mixed_pc_bf16"])
def test_block_cg_C_matches_oracle(femh, oracle, precision, kind):
    """Block PCG (block_cg=1: the six load cases of a cell share one Krylov
    space, the CG steps are 6x6 matrices from Cholesky solves of P^T K P and
    Z^T R) reaches the oracle's C^H and an FP64 residual below 1e-10 in every
    load case, in no more iterations than six independent PCG runs.  The
    laminate's zero right-hand sides stay out of the block, its equal ones
    (the in-plane normal strains load the layers alike) are dropped as
    dependent.  With store_bf16 the block keeps FP64 search directions."""
    rho = _block_cell(kind)
    Co = _oracle_C(oracle, "block_" + kind, rho)
    prec = femh.FP64 if precision == "fp64" else femh.MIXED_PC
    bf16 = 1 if precision == "mixed_pc_bf16" else 0
    C, info = femh.Engine(precision=prec, store_bf16=bf16, block_cg=1).homogenize(rho)
    assert info["status"] == 0 and max(info["rel_residual"]) < 1e-10
    assert _rel(C, Co) < (TOL_FP64 if precision == "fp64" else TOL_MIXED)
    C0, i0 = femh.Engine(precision=prec, block_cg=0).homogenize(rho)
    assert max(info["iterations"]) <= max(i0["iterations"])


@pytest.mark.parametrize("precision", ["fp64", "mixed_pc"])
def test_block_cg_batch_matches_single_cases(femh, precision):
    """A batch of uneven cells, each its own block: C^H equals the one-case
    PCG's within the solve tolerance, every cell converged, and no cell needs
    markedly more iterations than one-case PCG (the batch's unit lists shrink
    to the live cells as cells converge; the block's partial sums keep their
    slots)."""
    from fem_b200 import fields
    rhos = [fields.binary_cell(n, 0.3 + 0.05 * i, seed=60 + i) for i, n in enumerate((8, 16, 12, 24, 16, 32))]
    prec, tol = (femh.FP64, TOL_FP64) if precision == "fp64" else (femh.MIXED_PC, TOL_MIXED)
    Cb, infos, _ = femh.Engine(precision=prec, block_cg=1).batch(rhos, h=None)
    C0, infos0, _ = femh.Engine(precision=prec, block_cg=0).batch(rhos, h=None)
    for C, Cs, info, info0 in zip(Cb, C0, infos, infos0):
        assert info["status"] == 0 and max(info["rel_residual"]) < 1e-10
        assert _rel(C, Cs) < tol
        assert max(info["iterations"]) <= 1.2 * max(info0["iterations"]) + 5


_ORACLE_C = {}


def _oracle_C(oracle, key, rho):
    if key not in _ORACLE_C:
        _ORACLE_C[key] = oracle.homogenize(rho)[0]
    return _ORACLE_C[key]


@pytest.mark.parametrize("solver", ["jacobi", "gmg"])
@pytest.mark.parametrize("bf16", [0, 1])
def test_mixed_C_matches_oracle(femh, oracle, solver, bf16):
    from fem_b200 import fields
    rho = fields.smooth_cell(16, sigma=2.0, seed=2)
    Co, *_ = oracle.homogenize(rho)
    e = femh.Engine(precision=femh.MIXED, store_bf16=bf16,
                    solver=femh.JACOBI_PCG if solver == "jacobi" else femh.GMG_PCG)
    C, info = e.homogenize(rho)
    assert info["status"] == 0 and max(info["rel_residual"]) < 1e-10
    assert _rel(C, Co) < TOL_MIXED


@pytest.mark.parametrize("interp", ["simp", "ramp3", "binary"])
def test_material_laws(femh, oracle, interp):
    from fem_b200 import fields
    rho = fields.smooth_cell(8, sigma=1.5, seed=5)
    kw = {"simp": dict(interp=0), "ramp3": dict(interp=1, rho_min=1e-3),
          "binary": dict(interp=2, bin_hi=1.0, bin_lo=1e-4)}[interp]
    mat = oracle.material(interp=kw["interp"])
    rho_o = np.clip(rho, kw.get("rho_min", 0.0), 1.0)
    Co, *_ = oracle.homogenize(rho_o, mat=mat)
    e = femh.Engine(**kw)
    C, _ = e.homogenize(rho)
    assert _rel(C, Co) < TOL_FP64


def test_gradient_matches_oracle(femh, oracle):
    from fem_b200 import fields
    rho = fields.smooth_cell(12, sigma=2.0, seed=4)
    Co, chi_o, *_ = oracle.homogenize(rho, tol=1e-12)
    Ct = oracle.c_iso(0.05, 0.3)
    dLdC = 2 * (Co - Ct)
    go = oracle.grad(rho, chi_o, dLdC)
    e = femh.Engine(tol=1e-12)
    C, _ = e.homogenize(rho)
    g = e.grad(2 * (C - Ct))
    assert _rel(g, go) < TOL_GRAD
    d = e.dCdrho()
    do = oracle.dCdrho(rho, chi_o)
    assert _rel(d, do) < TOL_GRAD


def test_fluctuation_and_full_field(femh, oracle):
    """chi matches the oracle's (same pinned node), and the full-cell field is
    copyPeriodicU's: periodic chi plus eps.X with the jump on the + faces."""
    from fem_b200 import fields
    n = 8
    rho = fields.binary_cell(n, 0.6, seed=9)
    Co, chi_o, *_ = oracle.homogenize(rho, tol=1e-12)
    e = femh.Engine(tol=1e-12)
    e.homogenize(rho)
    chi = e.fluctuation()
    assert np.abs(chi - chi_o).max() < 1e-7 * np.abs(chi_o).max()
    h = 1.0 / n
    for I in range(6):
        u = e.full_field(I)
        eps = np.zeros((3, 3))
        if I < 3:
            eps[I, I] = 1
        else:
            a, b = [(1, 2), (0, 2), (0, 1)][I - 3]
            eps[a, b] = eps[b, a] = 0.5
        X = np.stack(np.meshgrid(*(np.arange(n + 1) * h,) * 3, indexing="ij"), -1)
        idx = np.arange(n + 1) % n
        ref = chi[I][np.ix_(idx, idx, idx)] + X @ eps.T
        assert np.abs(u - ref).max() < 1e-12


def test_batch_matches_single(femh):
    from fem_b200 import fields
    rhos = [fields.binary_cell(n, 0.4, seed=20 + n) for n in (8, 12, 16, 8, 24)]
    e = femh.Engine()
    Cb, infos, _ = e.batch(rhos, h=None)
    for r, C in zip(rhos, Cb):
        Cs, _ = femh.Engine().homogenize(r)
        assert _rel(C, Cs) < TOL_FP64


@pytest.mark.parametrize("precision", ["fp64", "mixed_pc"])
def test_batch_of_mixed_extents_matches_single(femh, precision):
    """Cells of several z extents with compile-time kernels in one batch: the
    level's stencil units are grouped by extent and each group launches its
    own kernel (here the staged ones, forced); every C^H equals that of a
    single-cell solve."""
    from fem_b200 import fields
    rhos = [fields.binary_cell(n, 0.45, seed=40 + i) for i, n in enumerate((16, 32, 24, 16, 48))]
    prec, var, tol = ((femh.FP64, 6, TOL_FP64) if precision == "fp64" else (femh.MIXED_PC, 5, TOL_MIXED))
    Cb, infos, _ = femh.Engine(precision=prec, stencil_variant=var).batch(rhos, h=None)
    for r, C, info in zip(rhos, Cb, infos):
        assert info["status"] == 0
        Cs, _ = femh.Engine(precision=prec).homogenize(r)
        assert _rel(C, Cs) < tol

