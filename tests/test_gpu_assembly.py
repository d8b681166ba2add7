"""Parity of the sm_100a tabulation and assembly kernels with the CPU oracle.

Matrices are compared on the same inputs with the same tabulation (the
oracle's table is handed to the GPU path through the tabulation cache file, the
way capytaine shares a table between runs), so the only differences left are
floating-point rounding: the bar is 1e-10 relative to the largest entry for the
float64 path and 2e-5 for the mixed-precision path.  Tables built on the GPU
are compared with the oracle's separately (float32 exp*E1 inside, 2e-8)."""
import os

import numpy as np
import pytest

from capytaine_b200.meshes import Mesh, mesh_sphere, mesh_rectangle, mesh_parallelepiped

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-10
MIXED_RTOL = 2e-5


def _gpu_gf(oracle_gf, tmp_path, **kwargs):
    """Product Green function reading the oracle's table from a cache file."""
    from capytaine_b200.green_function import Delhommeau
    gf = Delhommeau(tabulation_cache_dir=str(tmp_path), **kwargs)
    np.savez(os.path.join(str(tmp_path), gf._cache_filename), r_range=oracle_gf.tabulated_r_range,
             z_range=oracle_gf.tabulated_z_range, values=oracle_gf.tabulated_integrals)
    return gf


LEGACY = dict(tabulation_nr=328, tabulation_nz=46, tabulation_grid_shape="legacy",
              tabulation_nb_integration_points=251)


def _close(a, b, rtol):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max() / scale
    assert err <= rtol, f"max error {err:.3e} relative to max |entry| {scale:.3e}"


@pytest.mark.parametrize("legacy", [True, False])
def test_tabulation_built_on_gpu_matches_oracle(oracle_mod, legacy_oracle_gf, default_oracle_gf, legacy):
    from capytaine_b200.green_function import Delhommeau
    ora = legacy_oracle_gf if legacy else default_oracle_gf
    gf = Delhommeau(tabulation_cache_dir=None, **(LEGACY if legacy else {}))
    np.testing.assert_array_equal(gf.tabulated_r_range, ora.tabulated_r_range)
    np.testing.assert_array_equal(gf.tabulated_z_range, ora.tabulated_z_range)
    t_gpu = gf.tabulated_integrals
    t_ora = ora.tabulated_integrals
    for k in range(5):
        scale = np.abs(t_ora[..., k]).max()
        err = np.abs(t_gpu[..., k] - t_ora[..., k]).max() / scale
        assert err < 2e-8, (k, err)


CASES = {
    "hemisphere_lowfreq": dict(mesh=lambda: mesh_sphere(resolution=(10, 10)).immersed_part(), k=1.0, kw={}),
    "sphere_legacy_highfreq": dict(mesh=lambda: mesh_sphere(resolution=(6, 12)).immersed_part(), k=1 / 9.81,
                                   kw={}, legacy=True, sing="high_freq"),
    "full_gradient": dict(mesh=lambda: mesh_sphere(resolution=(8, 8)).immersed_part(), k=2.0,
                          kw=dict(early_dot_product=False)),
    "direct_D": dict(mesh=lambda: mesh_sphere(resolution=(8, 8)).immersed_part(), k=0.7,
                     kw=dict(adjoint_double_layer=False)),
    "direct_full_gradient": dict(mesh=lambda: mesh_sphere(resolution=(8, 8)).immersed_part(), k=0.7,
                                 kw=dict(adjoint_double_layer=False, early_dot_product=False)),
    "zero_frequency": dict(mesh=lambda: mesh_sphere(resolution=(8, 8)).immersed_part(), k=0.0, kw={}),
    "infinite_frequency": dict(mesh=lambda: mesh_sphere(resolution=(8, 8)).immersed_part(), k=np.inf, kw={}),
    "low_freq_with_rankine_part": dict(mesh=lambda: mesh_sphere(resolution=(8, 8)).immersed_part(), k=1.3,
                                       kw=dict(early_dot_product=False), sing="low_freq_with_rankine_part"),
    "barge_coarse": dict(mesh=lambda: mesh_parallelepiped(size=(8, 2, 2), resolution=(16, 4, 4)).immersed_part(),
                         k=3.0, kw={}),
    "gauss_legendre_2": dict(mesh=lambda: mesh_sphere(resolution=(6, 8)).immersed_part().with_quadrature(
        "Gauss-Legendre 2"), k=1.0, kw={}),
}


def _with_lid(mesh):
    lid = mesh_rectangle(size=(0.8, 0.8), resolution=(2, 2), center=(0, 0, 0), normal=(0, 0, 1))
    return Mesh.join_meshes(mesh, lid)


@pytest.mark.parametrize("name", sorted(CASES))
def test_assembly_fp64_matches_oracle(oracle_mod, legacy_oracle_gf, default_oracle_gf, tmp_path, name):
    case = CASES[name]
    mesh = case["mesh"]()
    legacy = case.get("legacy", False)
    sing = case.get("sing", "low_freq")
    settings = dict(LEGACY) if legacy else {}
    ora_base = legacy_oracle_gf if legacy else default_oracle_gf
    ora = oracle_mod.OracleDelhommeau(gf_singularities=sing, tabulation=ora_base.tabulation,
                                      tabulation_grid_shape=settings.get("tabulation_grid_shape", "scaled_nemoh3"),
                                      tabulation_nb_integration_points=settings.get(
                                          "tabulation_nb_integration_points", 1001))
    gf = _gpu_gf(ora_base, tmp_path, gf_singularities=sing, **settings)
    S_ref, K_ref = ora.evaluate(mesh, mesh, wavenumber=case["k"], **case["kw"])
    S, K = gf.evaluate(mesh, mesh, wavenumber=case["k"], **case["kw"])
    assert S.dtype == np.complex128 and K.dtype == np.complex128
    _close(S, S_ref, FP64_RTOL)
    _close(K, K_ref, FP64_RTOL)


def test_free_surface_panels(oracle_mod, default_oracle_gf, tmp_path):
    mesh = _with_lid(mesh_sphere(resolution=(6, 8)).immersed_part())
    gf = _gpu_gf(default_oracle_gf, tmp_path)
    for k in (0.5, 2.0):
        S_ref, K_ref = default_oracle_gf.evaluate(mesh, mesh, wavenumber=k)
        S, K = gf.evaluate(mesh, mesh, wavenumber=k)
        _close(S, S_ref, FP64_RTOL)
        _close(K, K_ref, FP64_RTOL)


def test_points_as_first_argument_and_asymptotic_branch(oracle_mod, default_oracle_gf, tmp_path):
    mesh = mesh_sphere(resolution=(6, 8)).immersed_part()
    rng = np.random.default_rng(0)
    pts = np.concatenate([rng.uniform(-3, 3, (40, 3)) * [1, 1, 0] + [0, 0, -0.5],
                          [[150.0, 0.0, -1.0], [0.0, 120.0, -300.0], [10.0, 10.0, -0.01]]])
    gf = _gpu_gf(default_oracle_gf, tmp_path)
    for kw in (dict(), dict(early_dot_product=False, diagonal_term_in_double_layer=False)):
        S_ref, K_ref = default_oracle_gf.evaluate(pts, mesh, wavenumber=1.0, **kw)
        S, K = gf.evaluate(pts, mesh, wavenumber=1.0, **kw)
        _close(S, S_ref, FP64_RTOL)
        _close(K, K_ref, FP64_RTOL)


def test_rankine_only(oracle_mod, default_oracle_gf, tmp_path):
    mesh = mesh_sphere(resolution=(8, 10))
    gf = _gpu_gf(default_oracle_gf, tmp_path)
    for kw in (dict(), dict(early_dot_product=False), dict(adjoint_double_layer=False)):
        S_ref, K_ref = default_oracle_gf.evaluate(mesh, mesh, free_surface=np.inf, **kw)
        S, K = gf.evaluate(mesh, mesh, free_surface=np.inf, **kw)
        assert not np.iscomplexobj(S)
        _close(S, S_ref, FP64_RTOL)
        _close(K, K_ref, FP64_RTOL)


def test_untabulated_direct_integration(oracle_mod):
    from capytaine_b200.green_function import Delhommeau
    mesh = mesh_sphere(resolution=(4, 6)).immersed_part()
    ora = oracle_mod.OracleDelhommeau(tabulation_nr=0, tabulation_nz=0, tabulation_nb_integration_points=101)
    gf = Delhommeau(tabulation_nr=0, tabulation_nz=0, tabulation_nb_integration_points=101, tabulation_cache_dir=None)
    S_ref, K_ref = ora.evaluate(mesh, mesh, wavenumber=1.5)
    S, K = gf.evaluate(mesh, mesh, wavenumber=1.5)
    # direct integration evaluates exp*E1 in float32 on both sides
    _close(S, S_ref, 1e-6)
    _close(K, K_ref, 1e-6)


def test_float32_outputs(oracle_mod, default_oracle_gf, tmp_path):
    mesh = mesh_sphere(resolution=(8, 8)).immersed_part()
    gf = _gpu_gf(default_oracle_gf, tmp_path, floating_point_precision="float32")
    S, K = gf.evaluate(mesh, mesh, wavenumber=1.0)
    assert S.dtype == np.complex64 and K.dtype == np.complex64
    S_ref, K_ref = default_oracle_gf.evaluate(mesh, mesh, wavenumber=1.0)
    _close(S, S_ref, 1e-6)
    _close(K, K_ref, 1e-6)


@pytest.mark.parametrize("k", [0.1, 1.0, 4.0])
def test_mixed_precision_assembly(oracle_mod, default_oracle_gf, tmp_path, k):
    mesh = mesh_parallelepiped(size=(10, 4, 4), resolution=(20, 8, 8)).immersed_part()
    gf = _gpu_gf(default_oracle_gf, tmp_path, precision="mixed")
    S_ref, K_ref = default_oracle_gf.evaluate(mesh, mesh, wavenumber=k)
    S, K = gf.evaluate(mesh, mesh, wavenumber=k)
    _close(S, S_ref, MIXED_RTOL)
    _close(K, K_ref, MIXED_RTOL)


def test_nan_is_reported(default_oracle_gf, tmp_path):
    from capytaine_b200 import _lib
    # two coincident panels: the collocation point sits on a vertex of the
    # other panel's twin, which yields NaN in the exact Rankine integral
    v = np.array([[0, 0, -1], [1, 0, -1], [1, 1, -1], [0, 1, -1]], dtype=float)
    mesh = Mesh(np.concatenate([v, v + [0.5, 0.5, 0]]), [[0, 1, 2, 3], [4, 5, 6, 7]], clean=False)
    gf = _gpu_gf(default_oracle_gf, tmp_path)
    with pytest.raises(_lib.GreenFunctionEvaluationError):
        gf.evaluate(mesh, mesh, wavenumber=1.0)


def test_golden_6x6_rankine_matrices(legacy_oracle_gf, golden, tmp_path):
    mesh = Mesh(np.array(golden["rankine_mesh_vertices"]), golden["rankine_mesh_faces"])
    gf = _gpu_gf(legacy_oracle_gf, tmp_path, gf_singularities="high_freq", **LEGACY)
    S, _ = gf.evaluate(mesh, mesh, water_depth=np.inf, wavenumber=0.0)
    assert np.allclose(S, golden["S_k0"])
    S, _ = gf.evaluate(mesh, mesh, water_depth=np.inf, wavenumber=np.inf)
    assert np.allclose(S, golden["S_kinf"])
