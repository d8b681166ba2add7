"""Host-side geometry of lids and multibodies: interior free-surface lids
(capytaine meshes/meshes.py:655-737) and joined bodies whose dofs act on their
own faces only (bodies/multibodies.py:34-122, bodies/dofs.py:100-127)."""
import numpy as np
import pytest

from capytaine_b200.bodies import FloatingBody, join_bodies, rigid_body_dofs
from capytaine_b200.meshes import mesh_parallelepiped, mesh_sphere, mesh_vertical_cylinder


def test_lid_of_a_vertical_cylinder():
    r = 5.0
    hull = mesh_vertical_cylinder(length=40, radius=r, resolution=(6, 48, 40)).immersed_part()
    lid = hull.generate_lid()
    assert lid.nb_faces > 0
    assert np.all(lid.vertices[:, 2] == 0.0)
    assert np.allclose(lid.faces_normals, [0.0, 0.0, -1.0])
    assert np.hypot(lid.vertices[:, 0], lid.vertices[:, 1]).max() <= r
    assert 0.5 * np.pi * r ** 2 < lid.faces_areas.sum() <= np.pi * r ** 2
    # panel size of the order of the mean face radius of the hull
    assert lid.faces_radiuses.max() <= 1.01 * np.mean(hull.faces_radiuses)


def test_lid_of_a_box_and_of_a_submerged_body():
    hull = mesh_parallelepiped(size=(8, 4, 4), resolution=(16, 8, 8)).immersed_part()
    lid = hull.generate_lid()
    assert np.all(np.abs(lid.vertices[:, 0]) <= 4.0) and np.all(np.abs(lid.vertices[:, 1]) <= 2.0)
    assert lid.faces_areas.sum() > 0.6 * 32.0
    deep = mesh_sphere(radius=1.0, center=(0, 0, -3), resolution=(8, 16))
    assert deep.generate_lid().nb_faces == 0


def test_joined_bodies_dofs_and_lids():
    bodies = []
    for i, (x, y) in enumerate([(0.0, 0.0), (30.0, 0.0), (0.0, 30.0)]):
        h = mesh_vertical_cylinder(length=20, radius=4, resolution=(3, 24, 10), center=(x, y, 0)).immersed_part()
        bodies.append(FloatingBody(h, rigid_body_dofs(rotation_center=(x, y, 0)), lid_mesh=h.generate_lid(),
                                   name=f"cyl{i}"))
    mb = join_bodies(*bodies)
    assert mb.name == "cyl0+cyl1+cyl2"
    assert list(mb.dofs)[:2] == ["cyl0__Surge", "cyl0__Sway"] and len(mb.dofs) == 18
    n_hull = [b.mesh.nb_faces for b in bodies]
    assert mb.mesh.nb_faces == sum(n_hull)
    assert mb.mesh_including_lid.nb_faces == sum(n_hull) + sum(b.lid_mesh.nb_faces for b in bodies)
    assert mb.hull_mask.sum() == sum(n_hull)
    d = mb.dof_normal_components()
    starts = np.cumsum([0] + n_hull)
    for j, name in enumerate(mb.dofs):
        body = int(name[3])
        on = np.zeros(d.shape[1], bool)
        on[starts[body]:starts[body + 1]] = True
        assert np.all(d[j, ~on] == 0.0)
        own = bodies[body].dof_normal_components()[j % 6]
        assert np.allclose(d[j, on], own[:n_hull[body]])
    assert (bodies[0] + bodies[1]).name == "cyl0+cyl1"
    with pytest.raises(ValueError):
        join_bodies(bodies[0], bodies[0])
