"""Lid generation against the reference's own tests
(pytest/test_meshes_lid_generation.py:31-127, the cases without gmsh)."""
import numpy as np

from capytaine_b200.meshes import mesh_parallelepiped, mesh_sphere, mesh_vertical_cylinder
from capytaine_b200.symmetric_meshes import ReflectionSymmetricMesh, RotationSymmetricMesh


def test_lid_below_free_surface():
    points = np.array([((z + 1.0) ** 2, 0, z) for z in np.linspace(-1.0, 0.0, 10)])
    mesh = RotationSymmetricMesh.from_profile_points(points, n=10).merged()
    lid = mesh.generate_lid(z=-0.5)
    x, y, z = lid.faces_centers.T
    assert lid.nb_faces > 0 and np.all(np.hypot(x, y) <= (z + 1.0) ** 2)


def test_lid_below_or_without_the_body():
    assert mesh_sphere(radius=0.5, center=(0, 0, 0.0)).generate_lid(z=-2.0).nb_vertices == 0
    assert mesh_sphere(radius=0.5, center=(0, 0, -1.5)).generate_lid().nb_vertices == 0


def test_lid_multibody():
    mesh = mesh_sphere(center=(0, 0, 0)).join_meshes(mesh_sphere(center=(0, 5, 0))).immersed_part()
    lid = mesh.generate_lid()
    x, y = lid.faces_centers[:, 0], lid.faces_centers[:, 1]
    assert lid.nb_faces > 0 and np.all((np.hypot(x, y) < 1.0) | (np.hypot(x, y - 5) < 1.0))


def test_lids_of_symmetric_meshes():
    lid = mesh_vertical_cylinder(radius=1, reflection_symmetry=True).immersed_part().generate_lid()
    assert isinstance(lid, ReflectionSymmetricMesh) and lid.nb_faces > 0
    assert np.all(np.hypot(lid.faces_centers[:, 0], lid.faces_centers[:, 1]) < 1.0)
    lid = mesh_parallelepiped(reflection_symmetry=True).immersed_part().generate_lid()
    assert isinstance(lid, ReflectionSymmetricMesh) and isinstance(lid.half, ReflectionSymmetricMesh)
    assert lid.nb_faces > 0 and np.all(np.maximum(np.abs(lid.faces_centers[:, 0]),
                                                  np.abs(lid.faces_centers[:, 1])) < 0.5)
    lid = mesh_vertical_cylinder(radius=0.5, axial_symmetry=True).immersed_part().generate_lid()
    assert isinstance(lid, RotationSymmetricMesh)
    assert np.all(np.hypot(lid.faces_centers[:, 0], lid.faces_centers[:, 1]) < 1.0)
