"""Radiation problems at zero and infinite frequency in the oracle, against
the reference's tests (pytest/test_bem_zero_and_infinite_freq.py:118-155):
a finite added mass and zero damping for a plain, a symmetric and a lidded
body, both methods, infinite depth; infinite frequency in finite depth; zero
frequency in finite depth refused.  The limits are also the limits of the
finite-frequency solve (omega -> 0 and omega -> large)."""
import numpy as np
import pytest

from capytaine_b200.bodies import FloatingBody
from capytaine_b200.meshes import mesh_parallelepiped, mesh_sphere


def _bodies():
    sphere = mesh_sphere(resolution=(4, 4)).immersed_part()
    box = mesh_parallelepiped(resolution=(2, 2, 2), reflection_symmetry=True).immersed_part()
    lidded = FloatingBody(sphere, lid_mesh=sphere.generate_lid())
    return {"simple": (sphere, None), "symmetric": (box.merged(), None),
            "lid": (lidded.mesh_including_lid, lidded.hull_mask)}


@pytest.mark.parametrize("kind", ["simple", "symmetric", "lid"])
@pytest.mark.parametrize("omega", [0.0, np.inf])
@pytest.mark.parametrize("method", ["direct", "indirect"])
def test_radiation_at_limit_frequencies(oracle_mod, default_oracle_gf, kind, omega, method):
    mesh, mask = _bodies()[kind]
    dofs = oracle_mod.rigid_body_dofs(only=["Surge"])
    r = oracle_mod.solve_radiation_limit_frequency(default_oracle_gf, mesh, dofs, omega, method=method,
                                                   hull_mask=mask)
    a = r["added_mass"]["Surge"]["Surge"]
    assert isinstance(a, float) and np.isfinite(a) and a > 0
    assert r["radiation_damping"]["Surge"]["Surge"] == 0.0


def test_finite_depth_limits(oracle_mod, default_oracle_gf):
    mesh, _ = _bodies()["simple"]
    dofs = oracle_mod.rigid_body_dofs(only=["Surge"])
    r = oracle_mod.solve_radiation_limit_frequency(default_oracle_gf, mesh, dofs, np.inf, water_depth=5.0)
    assert np.isfinite(r["added_mass"]["Surge"]["Surge"]) and r["radiation_damping"]["Surge"]["Surge"] == 0.0
    with pytest.raises(NotImplementedError):
        oracle_mod.solve_radiation_limit_frequency(default_oracle_gf, mesh, dofs, 0.0, water_depth=5.0)


def test_limits_of_the_finite_frequency_solve(oracle_mod, default_oracle_gf):
    """A(omega) tends to the limit values: at omega = 1e-3 the finite-frequency
    solve is within 1e-5 of the zero-frequency one (1.3e-6 measured); at
    omega = 60 (kr up to 370, where the panels no longer resolve the waves and
    the discretisation error dominates) within 1e-2 of the infinite-frequency
    one (2e-3 measured)."""
    mesh = mesh_sphere(resolution=(8, 16)).immersed_part()
    dofs = oracle_mod.rigid_body_dofs(only=["Heave"])
    for w_lim, w, rel in ((0.0, 1e-3, 1e-5), (np.inf, 60.0, 1e-2)):
        lim = oracle_mod.solve_radiation_limit_frequency(default_oracle_gf, mesh, dofs, w_lim)["added_mass"]
        fin = oracle_mod.solve_frequency(default_oracle_gf, mesh, dofs, w, wave_directions=())["added_mass"]
        assert fin["Heave"]["Heave"] == pytest.approx(lim["Heave"]["Heave"], rel=rel)
