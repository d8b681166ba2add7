"""The engine and Green-function seams on the host (no device call): settings
exported as capytaine's (pytest/test_bem_solver.py:32-61), rejected options,
the custom linear solver contract (pytest/test_bem_engines_basic_matrix_engine.py:
56-95) and the repr (:25-27)."""
import numpy as np
import pytest

from capytaine_b200.engine import B200Engine
from capytaine_b200.green_function import Delhommeau


def test_exportable_settings():
    gf = Delhommeau(tabulation_nr=10, tabulation_nz=10, tabulation_grid_shape="legacy",
                    tabulation_nb_integration_points=50, finite_depth_prony_decomposition_method="fortran",
                    tabulation_cache_dir=None)
    assert gf.exportable_settings["green_function"] == "Delhommeau"
    assert gf.exportable_settings["tabulation_nb_integration_points"] == 50
    assert gf.exportable_settings["tabulation_grid_shape"] == "legacy"
    assert gf.exportable_settings["finite_depth_prony_decomposition_method"] == "fortran"
    engine = B200Engine(green_function=gf)
    assert engine.exportable_settings["engine"] == "B200Engine"
    assert engine.exportable_settings["linear_solver"] == "lu_decomposition"
    assert engine.exportable_settings["tabulation_nb_integration_points"] == 50
    assert "Delhommeau" in repr(engine)
    assert hash(gf) == hash(Delhommeau(tabulation_nr=10, tabulation_nz=10, tabulation_grid_shape="legacy",
                                       tabulation_nb_integration_points=50,
                                       finite_depth_prony_decomposition_method="fortran", tabulation_cache_dir=None))


def test_rejected_options():
    gf = Delhommeau(tabulation_cache_dir=None)
    with pytest.raises(ValueError):
        B200Engine(green_function=gf, precision="half")
    with pytest.raises(NotImplementedError):
        B200Engine(green_function=gf, linear_solver="cholesky")
    with pytest.raises(ValueError):
        B200Engine(green_function=gf, precision="mixed", linear_solver="gmres")
    with pytest.raises(ValueError):
        B200Engine(green_function=gf, method="galerkin")
    with pytest.raises(ValueError):
        B200Engine(green_function=gf, refinement="newton")
    with pytest.raises(KeyError):
        Delhommeau(tabulation_grid_shape="unknown", tabulation_cache_dir=None)
    with pytest.raises(NotImplementedError):
        Delhommeau(floating_point_precision="float16", tabulation_cache_dir=None)


def test_custom_linear_solver_contract():
    gf = Delhommeau(tabulation_cache_dir=None)
    A = np.array([[2.0, 0.0], [0.0, 4.0]], dtype=complex)
    b = np.array([2.0, 4.0], dtype=complex)
    engine = B200Engine(green_function=gf, linear_solver=lambda A, b: np.linalg.solve(A, b))
    np.testing.assert_allclose(engine.linear_solver(A, b), [1.0, 1.0])
    assert engine.exportable_settings["linear_solver"].startswith("<function")
    wrong = B200Engine(green_function=gf, linear_solver=lambda A, b: np.ones(3))
    with pytest.raises(ValueError):
        wrong.linear_solver(A, b)


def test_tabulation_cache_file_name_is_the_reference_one():
    """delhommeau.py:221-225: a table cached by capytaine is read here and the
    other way round (same name, same npz keys r_range, z_range, values)."""
    assert Delhommeau(tabulation_cache_dir=None)._cache_filename == \
        "tabulation_float64_scaled_nemoh3_676_100.0_372_-251.0_1001.npz"
    gf = Delhommeau(tabulation_nr=3, tabulation_rmax=1, tabulation_nz=3, tabulation_zmin=-1,
                    tabulation_nb_integration_points=10, tabulation_grid_shape="legacy", tabulation_cache_dir=None)
    assert gf._cache_filename == "tabulation_float64_legacy_3_1.0_3_-1.0_10.npz"


@pytest.mark.parametrize("depth", [0.5, 1.0, 10.0, 1000.0])
def test_finite_depth_wavenumbers(oracle_mod, depth):
    """The dispersion relation omega^2 = g k tanh(k h) of the finite-depth
    problems (bem/problems_and_results.py:159-163; the reference's
    test_bem_problems_and_results.py:43-46 checks the same identity), against
    the oracle's root, from shallow to deep water."""
    from capytaine_b200.engine import wavenumbers
    omegas = np.array([1e-3, 0.05, 0.3, 1.0, 2.5, 8.0])
    ks = wavenumbers(omegas, depth)
    np.testing.assert_allclose(9.81 * ks * np.tanh(ks * depth), omegas ** 2, rtol=1e-14)
    ref = [oracle_mod.finite_depth_wavenumber(w, depth) for w in omegas]
    np.testing.assert_allclose(ks, ref, rtol=1e-12)
    assert np.all(ks >= omegas ** 2 / 9.81)  # tanh < 1: longer waves than in deep water


def test_infinite_depth_wavenumbers_and_limits():
    from capytaine_b200.engine import wavenumbers
    omegas = np.array([0.1, 1.0, 3.0])
    assert np.array_equal(wavenumbers(omegas), omegas ** 2 / 9.81)  # exactly, as the reference
    assert np.array_equal(wavenumbers(omegas, np.inf, 9.8), omegas ** 2 / 9.8)
    np.testing.assert_array_equal(wavenumbers([0.0, np.inf], 10.0), [0.0, np.inf])
    for depth in (0.0, -1.0, np.nan):
        with pytest.raises(ValueError):
            wavenumbers([1.0], depth)


def test_limit_frequency_coefficients():
    """At omega = 0 and infinity the forces come computed with omega = 1: the
    added mass is Re(F), the damping exactly zero and the wave forces NaN
    (capytaine's symbolic-frequency results, problems_and_results.py:583-592,
    airy_waves.py:36-37); finite omegas divide as usual."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.meshes import mesh_sphere
    body = FloatingBody(mesh_sphere(resolution=(4, 4)).immersed_part(), rigid_body_dofs(only=["Surge", "Heave"]))
    omegas = np.array([0.0, 2.0, np.inf])
    rng = np.random.default_rng(0)
    F = rng.standard_normal((3, 3, 2)) + 1j * rng.standard_normal((3, 3, 2))  # 2 dofs + 1 heading
    FK = rng.standard_normal((3, 1, 2)) + 1j * rng.standard_normal((3, 1, 2))
    res = B200Engine._coefficients(body, omegas, np.array([0.0]), F, FK, {})
    np.testing.assert_array_equal(res.added_mass[[0, 2]], F[[0, 2], :2].real)
    np.testing.assert_allclose(res.added_mass[1], F[1, :2].real / 4.0)
    assert np.all(res.radiation_damping[[0, 2]] == 0.0)
    np.testing.assert_allclose(res.radiation_damping[1], F[1, :2].imag / 2.0)
    assert np.all(np.isnan(res.excitation[[0, 2]])) and np.all(np.isnan(res.froude_krylov[[0, 2]]))
    np.testing.assert_allclose(res.excitation[1], F[1, 2:] + FK[1])
