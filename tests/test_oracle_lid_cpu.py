"""Lids for irregular-frequency removal in the oracle, against the reference's
own tests (pytest/test_bem_irregular_frequencies_removal.py:57-128): the lid
leaves the hull blocks of S, K and D unchanged, leaves the Froude-Krylov
force unchanged and changes the diffraction force at a regular frequency by
less than 5%."""
import numpy as np
import pytest

from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
from capytaine_b200.meshes import mesh_parallelepiped, mesh_rectangle


@pytest.fixture(scope="module")
def bodies():
    mesh = mesh_parallelepiped(center=(0.0, 0.0, -0.4)).immersed_part()
    lid = mesh_rectangle(size=(1, 1), resolution=(4, 4), center=(0, 0, 0), normal=(0, 0, -1))
    return FloatingBody(mesh, rigid_body_dofs()), FloatingBody(mesh, rigid_body_dofs(), lid_mesh=lid)


def test_lid_leaves_the_hull_blocks_unchanged(oracle_mod, default_oracle_gf, bodies):
    without, with_lid = bodies
    n = without.mesh.nb_faces
    full = with_lid.mesh_including_lid
    assert np.all(with_lid.hull_mask[:n]) and not np.any(with_lid.hull_mask[n:])
    for adjoint in (True, False):
        S_w, K_w = default_oracle_gf.evaluate(full, full, wavenumber=1.0, adjoint_double_layer=adjoint)
        S_o, K_o = default_oracle_gf.evaluate(without.mesh, without.mesh, wavenumber=1.0, adjoint_double_layer=adjoint)
        np.testing.assert_allclose(S_w[:n, :n], S_o, atol=1e-8)
        np.testing.assert_allclose(K_w[:n, :n], K_o, atol=1e-8)


@pytest.mark.parametrize("water_depth", [np.inf, 10.0])
def test_lid_and_the_forces(oracle_mod, default_oracle_gf, bodies, water_depth):
    without, with_lid = bodies
    dofs = oracle_mod.rigid_body_dofs(only=["Heave"])
    k = 2 * np.pi / 3.0  # wavelength 3 m
    omega = np.sqrt(9.81 * k * np.tanh(k * water_depth))
    r_o = oracle_mod.solve_frequency(default_oracle_gf, without.mesh, dofs, omega, water_depth=water_depth)
    r_w = oracle_mod.solve_frequency(default_oracle_gf, with_lid.mesh_including_lid, dofs, omega,
                                     hull_mask=with_lid.hull_mask, water_depth=water_depth)
    assert r_w["froude_krylov"][0.0]["Heave"] == pytest.approx(r_o["froude_krylov"][0.0]["Heave"])
    assert r_w["diffraction"][0.0]["Heave"] == pytest.approx(r_o["diffraction"][0.0]["Heave"], rel=5e-2)
