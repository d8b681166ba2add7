"""Two horizontal cylinders, with and without reflection symmetry and lids,
joined into one body (capytaine pytest/test_bodies_multibodies.py:232-268):
the joined meshes and masks have the sizes of the parts, lid faces sit on the
free surface, and the surge radiation force of the first cylinder at omega = 1
is the reference's 2151.7 + 54.053j within its 5% (oracle solve on the
joined faces with the hull mask); without lids, within 1e-4 (the digits the
reference prints)."""
import numpy as np
import pytest

from capytaine_b200.bodies import FloatingBody, join_bodies, rigid_body_dofs
from capytaine_b200.meshes import mesh_horizontal_cylinder


def _body(x, lid, sym, name):
    mesh = mesh_horizontal_cylinder(center=(x, 0, 0), reflection_symmetry=sym).immersed_part()
    return FloatingBody(mesh, rigid_body_dofs(rotation_center=(x, 0, 0)),
                        lid_mesh=mesh.generate_lid(faces_max_radius=0.3) if lid else None, name=name)


@pytest.mark.parametrize("lid_1,lid_2,sym_1,sym_2", [(False, False, False, False), (True, True, True, True),
                                                     (True, False, False, True), (False, True, True, False)])
def test_joined_cylinders_with_and_without_symmetry_and_lids(oracle_mod, default_oracle_gf, lid_1, lid_2, sym_1,
                                                             sym_2):
    b1, b2 = _body(0.0, lid_1, sym_1, "body_1"), _body(12.0, lid_2, sym_2, "body_2")
    for b in (b1, b2):
        assert b.hull_mask.shape == (b.mesh_including_lid.nb_faces,)
    both = join_bodies(b1, b2)
    assert both.mesh.nb_faces == b1.mesh.nb_faces + b2.mesh.nb_faces
    lids = [b.lid_mesh.nb_faces if b.lid_mesh is not None else 0 for b in (b1, b2)]
    assert (both.lid_mesh.nb_faces if both.lid_mesh is not None else 0) == sum(lids)
    assert both.mesh_including_lid.nb_faces == b1.mesh_including_lid.nb_faces + b2.mesh_including_lid.nb_faces
    assert both.hull_mask.shape[0] == b1.hull_mask.shape[0] + b2.hull_mask.shape[0]
    assert np.allclose(both.mesh_including_lid.faces_centers[~both.hull_mask, 2], 0.0)
    mask = np.zeros(both.mesh.nb_faces, bool)
    mask[:b1.mesh.nb_faces] = True
    surge = {"body_1__Surge": oracle_mod.SubmeshDof(oracle_mod.rigid_body_dofs()["Surge"], mask)}
    res = oracle_mod.solve_frequency(default_oracle_gf, both.mesh_including_lid, surge, 1.0, wave_directions=(),
                                     hull_mask=both.hull_mask if both.lid_mesh is not None else None)
    force = res["added_mass"]["body_1__Surge"]["body_1__Surge"] + 1j * res["radiation_damping"]["body_1__Surge"][
        "body_1__Surge"]  # omega = 1: F = A + i B
    assert force == pytest.approx(2151.7 + 54.053j, rel=0.05)
    if not (lid_1 or lid_2):  # the reference's number to its printed digits: 2151.79 + 54.057j here
        assert force == pytest.approx(2151.7 + 54.053j, rel=1e-4)
