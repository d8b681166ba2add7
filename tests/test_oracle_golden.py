"""Pins the CPU oracle against the reference's own known answers
(pytest/test_consistency_with_Nemoh_2.py, infinite and finite depth,
test_green_functions_fortran_core.py,
test_green_functions_table_density.py in the capytaine project)."""
import numpy as np
import pytest
from scipy.special import j0

from capytaine_b200.meshes import Mesh, mesh_sphere, mesh_rectangle
from conftest import hemisphere_volume


def test_rankine_and_reflected_rankine_6x6(legacy_oracle_gf, golden):
    # test_consistency_with_Nemoh_2.py:61-99
    mesh = Mesh(np.array(golden["rankine_mesh_vertices"]), golden["rankine_mesh_faces"])
    S, _ = legacy_oracle_gf.evaluate(mesh, mesh, water_depth=np.inf, wavenumber=0.0)
    assert np.allclose(S, golden["S_k0"])
    S, _ = legacy_oracle_gf.evaluate(mesh, mesh, water_depth=np.inf, wavenumber=np.inf)
    assert np.allclose(S, golden["S_kinf"])


@pytest.mark.parametrize("key,omega", [("omega_1", 1.0), ("omega_2", 2.0)])
def test_floating_sphere_nemoh2(legacy_oracle_gf, oracle_mod, golden, key, omega):
    # test_consistency_with_Nemoh_2.py:101-153
    sphere = mesh_sphere(radius=1.0, resolution=(6, 12)).immersed_part()
    ref = golden["floating_sphere"][key]
    atol = 1e-3 * hemisphere_volume(sphere) * 1000.0
    r = oracle_mod.solve_frequency(legacy_oracle_gf, sphere, oracle_mod.rigid_body_dofs(only=["Heave"]), omega)
    assert np.isclose(r["added_mass"]["Heave"]["Heave"], ref["added_mass"], atol=atol)
    assert np.isclose(r["radiation_damping"]["Heave"]["Heave"], ref["damping"], atol=atol)
    mod, phase = ref["diffraction_force_polar"]
    assert np.isclose(r["diffraction"][0.0]["Heave"], mod * np.exp(1j * phase), rtol=1e-3)


def test_alien_sphere(legacy_oracle_gf, oracle_mod, golden):
    # test_consistency_with_Nemoh_2.py:155-172
    ref = golden["alien_sphere"]
    sphere = mesh_sphere(radius=1.0, resolution=(6, 12)).immersed_part()
    atol = 1e-3 * hemisphere_volume(sphere) * ref["rho"]
    r = oracle_mod.solve_frequency(legacy_oracle_gf, sphere, oracle_mod.rigid_body_dofs(only=["Heave", "Surge"]),
                                   ref["omega"], rho=ref["rho"], g=ref["g"])
    assert np.isclose(r["added_mass"]["Heave"]["Heave"], ref["added_mass"], atol=atol)
    assert np.isclose(r["radiation_damping"]["Heave"]["Heave"], ref["damping"], atol=atol)
    mod, phase = ref["diffraction_force_polar"]
    assert np.isclose(r["diffraction"][0.0]["Heave"], mod * np.exp(1j * phase), rtol=1e-2)


@pytest.fixture(scope="module")
def legacy_finite_depth_gf(oracle_mod, legacy_oracle_gf):
    """The Nemoh 2 settings of the reference's finite-depth tests
    (test_consistency_with_Nemoh_2.py:23-33: legacy table, high_freq, legacy
    finite-depth method).  The reference decomposes with Nemoh's Fortran
    Prony routine there; the oracle uses capytaine's Python method, which
    meets the same tolerances."""
    return oracle_mod.OracleDelhommeau(tabulation_nr=328, tabulation_nz=46, tabulation_grid_shape="legacy",
                                       tabulation_nb_integration_points=251, gf_singularities="high_freq",
                                       finite_depth_method="legacy", tabulation=legacy_oracle_gf.tabulation)


@pytest.mark.parametrize("key,omega,tol_ab,tol_f", [("omega_1", 1.0, 1e-3, 1e-3), ("omega_2", 2.0, 1e-2, 1e-2)])
def test_floating_sphere_finite_depth_nemoh2(legacy_finite_depth_gf, oracle_mod, golden, key, omega, tol_ab, tol_f):
    # test_consistency_with_Nemoh_2.py:175-203, with the reference's tolerances
    ref = golden["floating_sphere_finite_depth"]
    sphere = mesh_sphere(radius=1.0, resolution=(6, 12)).immersed_part()
    atol = tol_ab * hemisphere_volume(sphere) * 1000.0
    r = oracle_mod.solve_frequency(legacy_finite_depth_gf, sphere, oracle_mod.rigid_body_dofs(only=["Heave"]), omega,
                                   water_depth=ref["depth"])
    assert np.isclose(r["added_mass"]["Heave"]["Heave"], ref[key]["added_mass"], atol=atol)
    assert np.isclose(r["radiation_damping"]["Heave"]["Heave"], ref[key]["damping"], atol=atol)
    mod, phase = ref[key]["diffraction_force_polar"]
    assert np.isclose(r["diffraction"][0.0]["Heave"], mod * np.exp(1j * phase), rtol=tol_f)


def test_two_distant_spheres_finite_depth_nemoh2(legacy_finite_depth_gf, oracle_mod, golden):
    # test_consistency_with_Nemoh_2.py:206-226: both spheres surge together
    ref = golden["two_spheres_finite_depth"]
    res = int(2 * np.pi * ref["radius"] * ref["resolution"])
    buoy = mesh_sphere(radius=ref["radius"], resolution=(res, res)).immersed_part()
    both, _ = buoy.join_meshes(buoy.translated((ref["spacing"], 0.0, 0.0)), return_masks=True)
    vol = 2 * 4 / 3 * np.pi * ref["radius"] ** 3
    r = oracle_mod.solve_frequency(legacy_finite_depth_gf, both, oracle_mod.rigid_body_dofs(only=["Surge"]),
                                   ref["omega"], water_depth=ref["depth"], wave_directions=())
    assert np.isclose(r["added_mass"]["Surge"]["Surge"], ref["added_mass_surge"], atol=1e-3 * vol * 1000.0)
    assert np.isclose(r["radiation_damping"]["Surge"]["Surge"], ref["damping_surge"], atol=1e-2 * vol * 1000.0)


def test_multibody_sphere_and_cylinder_nemoh2(legacy_oracle_gf, oracle_mod, golden):
    # test_consistency_with_Nemoh_2.py:228-270: a submerged sphere and a submerged
    # horizontal cylinder joined, surge and heave of each; the reference's table
    # has the influenced dof along rows and the radiating dof along columns
    from capytaine_b200.meshes import mesh_horizontal_cylinder
    ref = golden["multibody_sphere_cylinder"]
    cyl = mesh_horizontal_cylinder(length=5.0, radius=1.0, center=(1.5, 3, -3), resolution=(1, 10, 10))
    sph = mesh_sphere(radius=1.0, center=(0, 0, -2), resolution=(5, 20))
    both, (mc, ms) = cyl.join_meshes(sph, return_masks=True)
    dofs = {f"{b}__{d}": oracle_mod.SubmeshDof(oracle_mod.rigid_body_dofs()[d], mask)
            for b, mask in (("cylinder_1", mc), ("sphere_0", ms)) for d in ("Surge", "Heave")}
    assert list(dofs) == ref["dofs"]
    r = oracle_mod.solve_frequency(legacy_oracle_gf, both, dofs, ref["omega"], wave_directions=())
    atol = 1e-3 * (hemisphere_volume(cyl) + hemisphere_volume(sph)) * 1000.0
    A = np.array([[r["added_mass"][rad][inf] for rad in dofs] for inf in dofs])
    B = np.array([[r["radiation_damping"][rad][inf] for rad in dofs] for inf in dofs])
    np.testing.assert_allclose(A, ref["added_mass"], rtol=0, atol=atol)
    np.testing.assert_allclose(B, ref["damping"], rtol=0, atol=atol)
    # the oracle meets it with margin: 0.21 against the tolerance of 18
    np.testing.assert_allclose(A, ref["added_mass"], rtol=0, atol=0.5)


def test_immersed_sphere(legacy_oracle_gf, oracle_mod, golden):
    # test_consistency_with_Nemoh_2.py:36-58 (no free surface: Rankine kernel only)
    sphere = mesh_sphere(radius=1.0, resolution=(10, 40))
    vol = float(np.sum(sphere.faces_areas * sphere.faces_normals[:, 2] * sphere.faces_centers[:, 2]))
    atol = 1e-3 * vol * 1000.0
    dofs = oracle_mod.rigid_body_dofs(only=["Surge", "Heave"])
    r = oracle_mod.solve_frequency(legacy_oracle_gf, sphere, dofs, 1.0, free_surface=np.inf)
    assert np.isclose(r["added_mass"]["Heave"]["Heave"], golden["immersed_sphere"]["added_mass_heave"], atol=atol)
    assert np.isclose(r["added_mass"]["Surge"]["Surge"], golden["immersed_sphere"]["added_mass_surge"], atol=atol)
    assert np.isclose(r["added_mass"]["Heave"]["Surge"], 0.0, atol=atol)
    assert np.isclose(r["radiation_damping"]["Heave"]["Heave"], 0.0, atol=atol)


@pytest.mark.parametrize("nr,rmax,grid", [(324, 100.0, 0), (676, 100.0, 1), (600, 120.0, 1)])
def test_r_range_inversion(oracle_mod, nr, rmax, grid):
    # test_green_functions_table_density.py:130-142
    r_range = oracle_mod.default_r_spacing(nr, rmax, grid)
    assert np.all(r_range[:-1] < r_range[1:])
    idx = np.array([oracle_mod.nearest_r_index(r, r_range, grid) for r in r_range])
    if grid == 0:
        assert np.all(np.abs(idx - np.arange(1, nr + 1)) <= 1)
    else:
        assert np.all(idx == np.arange(1, nr + 1))


@pytest.mark.parametrize("nz,zmin,grid", [(46, -16.0, 0), (372, -251.0, 1)])
def test_z_range_inversion(oracle_mod, nz, zmin, grid):
    # test_green_functions_table_density.py:145-155
    z_range = oracle_mod.default_z_spacing(nz, zmin, grid)
    assert np.all(z_range[:-1] > z_range[1:])
    idx = np.array([oracle_mod.nearest_z_index(z, z_range, grid) for z in z_range])
    if grid == 0:
        assert np.all(np.abs(idx - np.arange(1, nz + 1)) <= 1)
    else:
        assert np.all(idx == np.arange(1, nz + 1))


def test_wave_part_variants_and_bessel_identity(default_oracle_gf):
    # test_green_functions_fortran_core.py:37-53
    gf = default_oracle_gf
    xi, xj, k = np.array([0.0, 0.0, -0.5]), np.array([0.0, 1.0, -0.5]), 2.0
    g_hf, _ = gf.wave_part_infinite_depth(xi, xj, k, "high_freq")
    g_lf, _ = gf.wave_part_infinite_depth(xi, xj, k, "low_freq")
    r = k * np.linalg.norm(xi[:2] - xj[:2])
    z = k * (xi[2] + xj[2])
    assert g_lf[0].real + 2 * k / np.hypot(r, z) == pytest.approx(g_hf[0].real, rel=1e-4)
    assert g_lf[0].imag == pytest.approx(g_hf[0].imag)
    assert g_lf[0].imag == pytest.approx(2 * np.pi * k * np.exp(z) * j0(r), rel=1e-4)


@pytest.mark.parametrize("sing", ["low_freq", "high_freq"])
def test_wave_part_finite_differences(default_oracle_gf, sing):
    # test_green_functions_fortran_core.py:56-79
    gf = default_oracle_gf
    k, xi, xj = 1.0, np.array([0.0, 0.0, -0.5]), np.array([1.0, 1.0, -0.5])
    g0, nabla = gf.wave_part_infinite_depth(xi, xj, k, sing)
    fd = []
    for e in np.eye(3) * 1e-3:
        g1, _ = gf.wave_part_infinite_depth(xi + e, xj, k, sing)
        fd.append((g1[0] - g0[0]) / 1e-3)
    assert nabla[0] == pytest.approx(np.array(fd), abs=1e-2)


def test_wave_part_value(default_oracle_gf):
    # test_green_functions_fortran_core.py:82-92
    g, nabla = default_oracle_gf.wave_part_infinite_depth([0.0, 0.0, -0.5], [1.0, 1.0, -0.5], 1.0, "low_freq")
    assert g[0] == pytest.approx(-2.04 + 1.29j, abs=0.1)
    assert nabla[0] == pytest.approx([0.25 + 0.88j, 0.25 + 0.88j, -0.88 + 1.29j], abs=0.1)


def test_wave_part_symmetry(legacy_oracle_gf):
    # test_green_functions_fortran_core.py:101-114
    xi, xj = np.array([0.0, 0.0, -1.0]), np.array([1.0, 1.0, -2.0])
    for sing in ("high_freq", "low_freq"):
        g1, d1 = legacy_oracle_gf.wave_part_infinite_depth(xi, xj, 1.0, sing)
        g2, d2 = legacy_oracle_gf.wave_part_infinite_depth(xj, xi, 1.0, sing)
        assert g1[0] == pytest.approx(g2[0])
        assert d1[0][:2] == pytest.approx(-d2[0][:2])
        assert d1[0][2] == pytest.approx(d2[0][2])


def test_exact_rankine_additivity(default_oracle_gf):
    # test_green_functions_fortran_core.py:142-151
    c = np.zeros((1, 3))
    once = default_oracle_gf.evaluate_rankine_only(c, mesh_rectangle(size=(1, 1), resolution=(1, 1)),
                                                   diagonal_term_in_double_layer=False)[0]
    parts = default_oracle_gf.evaluate_rankine_only(c, mesh_rectangle(size=(1, 1), resolution=(11, 11)),
                                                    diagonal_term_in_double_layer=False)[0]
    assert once[0, 0] == pytest.approx(parts.sum(), abs=1e-2)


def test_rankine_alone_vs_zero_and_infinite_frequency(default_oracle_gf):
    # test_green_functions_fortran_core.py:154-173
    gf = default_oracle_gf
    p = np.array([[1.0, 0.0, -1.0]])
    pm = np.array([[1.0, 0.0, 1.0]])
    mesh = mesh_rectangle(size=(1.0, 1.0), center=(0.0, 0.0, -1.0), resolution=(1, 1))
    a = gf.evaluate_rankine_only(p, mesh)[0] + gf.evaluate_rankine_only(pm, mesh)[0]
    assert a == pytest.approx(gf.evaluate(p, mesh, wavenumber=0.0)[0])
    b = gf.evaluate_rankine_only(p, mesh)[0] - gf.evaluate_rankine_only(pm, mesh)[0]
    assert b == pytest.approx(gf.evaluate(p, mesh, wavenumber=np.inf)[0])


def test_tabulated_vs_untabulated(oracle_mod, default_oracle_gf):
    # test_green_functions_fortran_core.py:122-126
    mesh = mesh_sphere(resolution=(6, 6)).immersed_part()
    untab = oracle_mod.OracleDelhommeau(tabulation_nr=0, tabulation_nz=0)
    assert np.allclose(untab.evaluate(mesh, mesh)[0], default_oracle_gf.evaluate(mesh, mesh)[0], atol=1e-2)


def test_layout_equivalences(default_oracle_gf):
    # test_green_functions_matrix_shape.py:23-97
    mesh = mesh_sphere(resolution=(4, 4)).immersed_part()
    gf = default_oracle_gf
    for adjoint in (True, False):
        _, gradG = gf.evaluate(mesh, mesh, wavenumber=1.0, early_dot_product=False, adjoint_double_layer=adjoint)
        _, K = gf.evaluate(mesh, mesh, wavenumber=1.0, early_dot_product=True, adjoint_double_layer=adjoint)
        spec = "kij,ik->ij" if adjoint else "kij,jk->ij"
        np.testing.assert_allclose(K, np.einsum(spec, gradG, mesh.faces_normals), atol=1e-12)
        _, g0 = gf.evaluate(mesh, mesh, wavenumber=1.0, early_dot_product=False, adjoint_double_layer=adjoint,
                            diagonal_term_in_double_layer=False)
        diag = np.zeros_like(gradG)
        for i in range(mesh.nb_faces):
            diag[:, i, i] = mesh.faces_normals[i]
        np.testing.assert_allclose(g0, gradG - 0.5 * diag, atol=1e-10, rtol=1e-10)


def test_direct_and_indirect_methods_agree(oracle_mod, default_oracle_gf):
    # test_bem_solver.py:24-83: coarse sphere, surge diffraction force at omega = 1, rel 1e-1;
    # the two formulations converge slowly with the mesh (5.6%, 7.4%, 4.2% apart at 4x4,
    # 10x20, 20x40 panels), so the finer mesh and the finite-depth case keep the same bound
    dofs = oracle_mod.rigid_body_dofs(only=["Surge"])
    for resolution, depth, rel in (((4, 4), np.inf, 1e-1), ((10, 20), np.inf, 1e-1), ((10, 20), 5.0, 1e-1)):
        sphere = mesh_sphere(radius=1.0, resolution=resolution).immersed_part()
        d = oracle_mod.solve_frequency(default_oracle_gf, sphere, dofs, 1.0, method="direct", water_depth=depth)
        i = oracle_mod.solve_frequency(default_oracle_gf, sphere, dofs, 1.0, method="indirect", water_depth=depth)
        assert d["diffraction"][0.0]["Surge"] == pytest.approx(i["diffraction"][0.0]["Surge"], rel=rel)
