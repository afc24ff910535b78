"""GPU test of the reference-facing C++ layer (fem_b200/host): the C++ program
tests/cpp/test_host.cpp drives FEM3DFun and NumericalCoarseningUsingMultigrid
like the reference's callers do; its outputs are checked here against the
oracle and against finite differences."""
import json
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def host_out(femh, tmp_path_factory):
    work = tmp_path_factory.mktemp("cpp")
    exe = str(work / "test_host")
    lib = os.path.join(ROOT, "fem_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-o", exe, os.path.join(ROOT, "tests", "cpp", "test_host.cpp"),
                    f"-L{lib}", "-lfemh", f"-Wl,-rpath,{lib}"], check=True)
    res = subprocess.run([exe, str(work)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    return json.loads(res.stdout)


def test_fem3dfun_G_matches_oracle(host_out, oracle):
    n = 8
    x0 = np.array(host_out["x0"]).reshape(n, n, n)
    rho = np.clip(x0, 1e-3, 1.0)
    Co, *_ = oracle.homogenize(rho, mat=oracle.material(interp=oracle.INTERP_RAMP3, E_s=1.0))
    G = np.array(host_out["G"]).reshape(6, 6)
    assert np.abs(G - Co).max() < 1e-8 * np.abs(Co).max()
    assert host_out["density"] == pytest.approx(rho.mean(), rel=1e-12)


def test_fem3dfun_df_matches_central_differences(host_out):
    fd = np.array(host_out["df_fd"])
    an = np.array(host_out["df_adjoint"])
    assert np.abs(fd - an).max() <= 1e-5 * np.abs(an).max()


def test_coarsening_outputs(host_out, oracle):
    tv = np.array(host_out["coarsened_tensors"])
    pv = np.array(host_out["coarsened_params"])
    assert tv.size == 63 and pv.size == 12 and host_out["batch_max_diff"] < 1e-9
    # structure 0, replicated once, subdivided twice -> 8^3 cell, two-material law
    s0 = np.array(host_out["struct0"]).reshape(4, 4, 4)
    cells = np.repeat(np.repeat(np.repeat(s0, 2, 0), 2, 1), 2, 2)
    mu1, lam1 = 1.0 / 2.6, 0.3 / (1.3 * 0.4)
    E1 = mu1 * (3 * lam1 + 2 * mu1) / (lam1 + mu1)
    nu1 = lam1 / (2 * (lam1 + mu1))
    mat = oracle.material(interp=oracle.INTERP_BINARY, bin_hi=E1, bin_lo=E1 * 1e-4, nu=nu1)
    Co, *_ = oracle.homogenize(cells.astype(float), mat=mat)
    lower = np.array([Co[i, j] for i in range(6) for j in range(i + 1)])
    assert np.abs(tv[:21] - lower).max() < 1e-8 * np.abs(lower).max()
    r, E, nu, G = pv[:4]
    a = Co[0, 1] / Co[0, 0]
    assert r == pytest.approx(s0.mean(), rel=1e-12)
    assert nu == pytest.approx(a / (1 + a), rel=1e-8)
    assert G == pytest.approx(Co[3, 3], rel=1e-8)


def test_force_driven_coarsening_outputs(host_out, oracle):
    """femh_host::NumericalCoarsening (femlib's force-driven class) against the
    oracle's restatement of femlib's multiplier system on structure 0 (8^3 after
    subdivision): the 21 tensor values and (rho, Y, nu_xy, G) within the FP64
    bar; the batched call equals the one-at-a-time call; General gives three
    Y, three nu, three G; a non-cubic cell is rejected."""
    from oracle import femlib_force as ff
    tv = np.array(host_out["force_tensors"])
    pv = np.array(host_out["force_params"])
    assert tv.size == 63 and pv.size == 12 and host_out["force_batch_max_diff"] < 1e-9
    assert host_out["force_noncubic_rejected"]
    s0 = np.array(host_out["struct0"]).reshape(4, 4, 4)
    cells = np.repeat(np.repeat(np.repeat(s0, 2, 0), 2, 1), 2, 2).astype(int)
    lame = [(0.1, 0.15), (1.0 / 2.6, 0.3 / (1.3 * 0.4))]
    E = [mu * (3 * lam + 2 * mu) / (lam + mu) for mu, lam in lame]
    nu = lame[1][1] / (2 * (lame[1][1] + lame[1][0]))
    C, lower, params = ff.coarsen(cells.ravel(), (8, 8, 8), E, nu, mats_in=s0.ravel().astype(int),
                                  regularize=False)
    assert np.abs(tv[:21] - lower).max() < 1e-8 * np.abs(lower).max()
    assert np.abs(pv[:4] - params).max() < 1e-8 * np.abs(params).max()
    _, _, pg = ff.coarsen(cells.ravel(), (8, 8, 8), E, nu, mats_in=s0.ravel().astype(int), cubic=False,
                          regularize=False)
    assert np.abs(np.array(host_out["force_params_general"]) - pg).max() < 1e-8 * np.abs(pg).max()


def test_binary_roundtrip(host_out):
    assert host_out["binary_roundtrip"] and host_out["fails"] == 0


def test_gradient_descent_decreases_objective(host_out):
    """femh_host::gradientDescent (fast_fem/run3d.cpp:268-289 restated) on the
    FEM3DFun objective: at least one accepted step, f strictly lower."""
    f0, f1 = host_out["descent_f"]
    assert host_out["descent_steps"] >= 1 and f1 < f0


def test_fem3dfun_matches_reference_fast_fem(host_out):
    """femh_host::FEM3DFun (GPU solve, energy and adjoint) against the
    reference's own fast_fem FEM3DFun (fast_fem/FEM3DFun.cpp:128-268, built by
    oracle/build_ref.sh with the oracle's solve behind stand-in topoOptLib
    headers) on an 8^3 cell over a 4^3 field, a PiecewiseConstant3D one and
    run3D's PiecewiseConstantCubic3D one: the upper triangle of G (the part the
    reference fills) and f within the FP64 bar 1e-8, df within 1e-8."""
    from oracle import ref as R
    if not R.available("libfastfem_ref.so"):
        pytest.skip("oracle/_ref/libfastfem_ref.so not built")
    G0 = np.array(host_out["ff_G0"]).reshape(6, 6)
    wG = np.array(host_out["ff_wG"]).reshape(6, 6)
    r = R.fastfem(8, np.array(host_out["ff_x0"]), 0.3, G0, wG, 0.4, 0.1)
    assert r["status"] == 0
    G = np.array(host_out["ff_G"]).reshape(6, 6)
    iu = np.triu_indices(6)
    assert np.abs(G[iu] - r["G"][iu]).max() < 1e-8 * np.abs(r["G"]).max()
    assert host_out["ff_f"] == pytest.approx(r["f"], rel=1e-8)
    df = np.array(host_out["ff_df"])
    assert np.abs(df - r["df"]).max() < 1e-8 * np.abs(r["df"]).max()
    # run3D's cubic-symmetric field: the chain rule on the device (femh_field_gradient)
    rc = R.fastfem(8, np.array(host_out["ff_x0"]), 0.3, G0, wG, 0.4, 0.1, kind=R.FIELD_CUBIC)
    assert rc["status"] == 0
    Gc = np.array(host_out["ffc_G"]).reshape(6, 6)
    assert np.abs(Gc[iu] - rc["G"][iu]).max() < 1e-8 * np.abs(rc["G"]).max()
    assert host_out["ffc_f"] == pytest.approx(rc["f"], rel=1e-8)
    dfc = np.array(host_out["ffc_df"])
    assert np.abs(dfc - rc["df"]).max() < 1e-8 * np.abs(rc["df"]).max()


def test_force_driven_coarsening_matches_reference_code(host_out):
    """femh_host::NumericalCoarsening against the reference's own
    NumericalCoarsening (SamplesGenerator/NumericalCoarsening.cpp:266-340, built
    as shipped -- float, 1 + 1e-5 diagonal scaling -- with Eigen's LU for the
    absent PARDISO) on structure 0 subdivided to 8^3: the 21 tensor values and
    (rho, Y, nu_xy, G): tensor within 1e-4, parameters within 3e-4 relative.
    The engine returns the exact, unscaled values; the reference's 1 + 1e-5
    diagonal scaling moves Y on this cell by 1.2e-4 (the scaled restatement
    matches the reference to 2e-5, tests/test_ref_pins.py), its float
    arithmetic by ~1e-6."""
    from oracle import ref as R
    if not R.available("libnc_ref.so"):
        pytest.skip("oracle/_ref/libnc_ref.so not built")
    s0 = np.array(host_out["struct0"]).reshape(4, 4, 4)
    cells = np.repeat(np.repeat(np.repeat(s0, 2, 0), 2, 1), 2, 2).astype(np.int32)
    lame = [(0.1, 0.15), (1.0 / 2.6, 0.3 / (1.3 * 0.4))]
    E = [mu * (3 * lam + 2 * mu) / (lam + mu) for mu, lam in lame]
    nu = lame[1][1] / (2 * (lame[1][1] + lame[1][0]))
    tv, pv = R.nc_coarsen(cells, E, nu, (0.0, 1.0), R.CUBIC)
    assert np.abs(np.array(host_out["force_tensors"])[:21] - tv).max() < 1e-4 * np.abs(tv).max()
    assert np.abs(np.array(host_out["force_params"])[:4] - pv).max() < 3e-4 * np.abs(pv).max()
