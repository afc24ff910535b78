"""The C++ host layer's own logic on the CPU (no GPU): fem_b200/host/femh_host.cpp
linked against tests/cpp/fake_femh.cpp, a stand-in for the engine's C ABI that
returns deterministic tensors.  Every output of tests/cpp/test_host_logic.cpp
is recomputed here from those tensors: femlib's force-driven parameters
(Y_a = A_a / S_aa, nu_ab = -S_ba / S_aa, G_i = C(3+i, 3+i), rho = mean base
density; SamplesGenerator/NumericalCoarsening.cpp:300-339), the multigrid
class's (rho, E, nu, G) (NumericalCoarseningUsingMultiGrid.cpp:326-339), the
material mapping, and FEM3DFun's objective and chain rule
(fast_fem/FEM3DFun.cpp:128-268)."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LAME = [(0.1, 0.15), (1.0 / 2.6, 0.3 / (1.3 * 0.4))]
STRUCTS = [[0, 1, 1, 0, 1, 0, 0, 1], [1, 1, 1, 0, 1, 1, 0, 1], [0, 0, 1, 0, 0, 1, 0, 0]]
DENS = [0.1, 0.9]


@pytest.fixture(scope="module")
def out(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("hostlogic") / "test_host_logic")
    cpp = os.path.join(ROOT, "tests", "cpp")
    subprocess.run(["g++", "-std=c++17", "-O1", "-o", exe, os.path.join(cpp, "test_host_logic.cpp"),
                    os.path.join(cpp, "fake_femh.cpp"), os.path.join(ROOT, "fem_b200", "host", "femh_host.cpp")],
                   check=True)
    r = subprocess.run([exe], capture_output=True, text=True, check=True, timeout=60)
    return json.loads(r.stdout)


def _young(mu, lam):
    return mu * (3 * lam + 2 * mu) / (lam + mu), lam / (2 * (lam + mu))


def _fake_C(E, nu):
    """tests/cpp/fake_femh.cpp's C^H of a cell of mean modulus E."""
    lam, mu = E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[[0, 1, 2], [0, 1, 2]] += 2 * mu
    C[[3, 4, 5], [3, 4, 5]] = mu
    C[0, 0] *= 1.05
    C[1, 1] *= 1.03
    C[3, 3] *= 1.02
    return C


def _lower(C):
    return np.array([C[i, j] for i in range(6) for j in range(i + 1)])


def test_force_driven_class(out):
    (E0, nu0), (E1, nu1) = _young(*LAME[0]), _young(*LAME[1])
    assert nu0 == pytest.approx(nu1)
    tv = np.array(out["force_tensors"]).reshape(3, 21)
    pv = np.array(out["force_params"]).reshape(3, 4)
    for s, t, p in zip(STRUCTS, tv, pv):
        s = np.array(s)
        C = _fake_C(np.where(s == 1, E1, E0).mean(), nu1)
        Cf = C * np.outer([1, 1, 1, .9, .9, .9], [1, 1, 1, .9, .9, .9])
        S = np.linalg.inv(C)
        assert np.allclose(t, _lower(Cf), rtol=1e-13, atol=0)
        # 4^3 cell spanning the unit cube: unit face areas
        assert np.allclose(p, [np.mean(np.array(DENS)[s]), 1 / S[0, 0], -S[1, 0] / S[0, 0], Cf[3, 3]],
                           rtol=1e-12, atol=0)
    assert out["force_tensors_batch"] == out["force_tensors"]
    assert out["force_params_batch"] == out["force_params"]
    s = np.array(STRUCTS[0])
    C = _fake_C(np.where(s == 1, E1, E0).mean(), nu1)
    Cf = C * np.outer([1, 1, 1, .9, .9, .9], [1, 1, 1, .9, .9, .9])
    S = np.linalg.inv(C)
    general = [np.mean(np.array(DENS)[s]), 1 / S[0, 0], 1 / S[1, 1], 1 / S[2, 2], -S[1, 0] / S[0, 0],
               -S[2, 0] / S[0, 0], -S[2, 1] / S[1, 1], Cf[3, 3], Cf[4, 4], Cf[5, 5]]
    assert np.allclose(out["force_params_general"], general, rtol=1e-12, atol=0)
    # repMaterialAssignment with two subdivisions = repetition along every axis
    cell0 = np.array(STRUCTS[0]).reshape(2, 2, 2).repeat(2, 0).repeat(2, 1).repeat(2, 2)
    assert np.array_equal(np.array(out["cell0"]).reshape(4, 4, 4), cell0)


def test_batches_split_by_node_budget(out):
    """computeBatch splits the structures into engine calls of at most
    maxNodesPerCall voxels, or by default into calls that fit the device
    (femh_batch_memory's estimate against 92% of the available memory), and
    returns the same values as one call."""
    assert out["force_split_calls"] == 3 and out["force_split_equal"]
    assert out["force_auto_calls"] == 2 and out["force_auto_equal"]
    assert out["mg_split_calls"] == 2 and out["mg_split_equal"]


def test_failed_batch_leaves_outputs_unchanged(out):
    """A part of a split batch that fails (FEMH_E_OOM from the engine) raises
    and appends nothing: the caller can retry with a smaller budget without
    duplicate tensors."""
    assert out["force_failed_code"] == 3 and out["force_failed_untouched"]
    assert out["mg_failed_code"] == 3 and out["mg_failed_untouched"]


def test_multigrid_reference_lower_triangle_switch(out):
    """referenceLowerTriangle = true appends what the reference's tensor files
    hold -- C(i, j), j <= i, of a C whose lower triangle it never fills
    (SamplesGenerator/NumericalCoarseningUsingMultiGrid.cpp:296-324): the 15
    off-diagonal values are 0, the diagonal ones and the parameters unchanged.
    The default appends the symmetric tensor's values."""
    ref = np.array(out["mg_tensors_reference_triangle"])
    full = np.array(out["mg_tensors"])
    diag = [t for t, (i, j) in enumerate((i, j) for i in range(6) for j in range(i + 1)) if i == j]
    off = [t for t in range(21) if t not in diag]
    assert np.all(ref[off] == 0.0) and np.any(full[off] != 0.0)
    assert np.array_equal(ref[diag], full[diag])
    assert out["mg_params_reference_triangle"] == out["mg_params"]


def test_force_driven_argument_errors(out):
    assert out["err_noncubic"] == 1        # FEMH_E_ARG from femh_force_tensors
    assert out["err_material_index"] == 1  # indices other than 0 / 1
    assert out["err_nu_mismatch"] == 1     # base materials of different Poisson ratios
    assert out["err_void"] == 1            # zero-stiffness base material
    assert out["err_uninitialised"] == 6   # FEMH_E_STATE before init()


def test_multigrid_class_parameters(out):
    """Material 1 -> E1, others E1 * 1e-4 (the density floor); (rho, E, nu, G)."""
    E1, nu1 = _young(*LAME[1])
    s = np.array(STRUCTS[0])
    C = _fake_C(np.where(s == 1, E1, E1 * 1e-4).mean(), nu1)
    assert np.allclose(out["mg_tensors"], _lower(C), rtol=1e-13, atol=0)
    a = C[0, 1] / C[0, 0]
    nu = a / (1 + a)
    E = C[0, 1] * (1 + nu) * (1 - 2 * nu) / nu
    assert np.allclose(out["mg_params"], [np.mean(np.array(DENS)[s]), E, nu, C[3, 3]], rtol=1e-12, atol=0)


def test_fem3dfun_objective_and_chain_rule(out):
    x0 = np.array(out["fun_x0"])
    dist = np.clip(x0.reshape(2, 2, 2).repeat(2, 0).repeat(2, 1).repeat(2, 2), 1e-3, 1.0)
    assert np.allclose(np.array(out["fun_distribution"]).reshape(4, 4, 4), dist, rtol=0, atol=0)
    density = dist.mean()
    assert out["fun_density"] == pytest.approx(density, rel=1e-14)
    G = _fake_C((2.0 * dist / (3 - 2 * dist)).mean(), 0.25)   # RAMP3 law, E = 2, nu = 0.25
    assert np.allclose(np.array(out["fun_G"]).reshape(6, 6), G, rtol=1e-13, atol=1e-16)
    idx = np.arange(36)
    wG = (1.0 + 0.1 * (idx % 7)).reshape(6, 6)
    G0 = np.where(idx % 7 == 0, 0.3, 0.01).reshape(6, 6)
    f = 0.5 * np.sum(wG * (G - G0) ** 2) + 0.5 * 0.7 * (density - 0.4) ** 2
    assert out["fun_f"] == pytest.approx(f, rel=1e-13)
    # dL/drho_e of the fake engine = trace(dL/dC); plus the volume term; summed
    # over the 2x2x2 voxels of each field parameter
    g = np.trace(wG * (G - G0)) + 0.7 / 64 * (density - 0.4)
    assert np.allclose(out["fun_df"], 8 * g, rtol=1e-13, atol=0)


def test_symmetric_field_maps_match_reference(out):
    """femh_host::PiecewiseConstantSym3D / Cubic3D assign every voxel centre of
    a 7x8x9 grid the same parameter as the reference's own field classes
    (fast_fem/PiecewiseConstantSym3D.cpp, PiecewiseConstantCubic3D.cpp, built
    by oracle/build_ref.sh); the maps feed femh_field_gradient."""
    from oracle import ref as R
    if not R.available("libfastfem_ref.so"):
        pytest.skip("oracle/_ref/libfastfem_ref.so not built")
    n = (7, 8, 9)
    for key, kind in (("map_sym", R.FIELD_SYM), ("map_cubic", R.FIELD_CUBIC)):
        got = np.array(out[key]).astype(int)
        want = [R.field_index(kind, 3, ((i + .5) / n[0], (j + .5) / n[1], (k + .5) / n[2]))
                for i in range(n[0]) for j in range(n[1]) for k in range(n[2])]
        assert np.array_equal(got, want), key
    assert len(set(np.array(out["map_cubic"]).astype(int))) < len(set(np.array(out["map_sym"]).astype(int)))
