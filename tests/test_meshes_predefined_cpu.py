"""Mesh generators against the reference's own generator tests
(pytest/test_meshes_predefined.py): panel counts, positions, symmetries,
maximal panel radius and rejected inputs."""
import numpy as np
import pytest

from capytaine_b200.meshes import (Mesh, mesh_disk, mesh_horizontal_cylinder, mesh_parallelepiped, mesh_rectangle,
                                   mesh_sphere, mesh_vertical_cylinder)
from capytaine_b200.symmetric_meshes import ReflectionSymmetricMesh, RotationSymmetricMesh


def _outward(mesh):
    c = mesh.faces_centers
    return np.min(np.sum((c - c.mean(axis=0)) * mesh.faces_normals, axis=1)) > 0


def test_disk():
    """test_meshes_predefined.py:27-59"""
    d = mesh_disk(resolution=(3, 6), name="foo")
    assert isinstance(d, Mesh) and d.nb_faces == 18 and d.name == "foo"
    d = mesh_disk(center=(1.0, 0.5, -0.5), normal=(0, 1, 0))
    assert np.allclose(d.vertices[:, 1], 0.5)
    assert np.allclose(d.faces_normals, (0, 1, 0))
    d = mesh_disk(resolution=(3, 6), reflection_symmetry=True)
    assert isinstance(d, ReflectionSymmetricMesh) and np.all(d.half.vertices[:, 1] >= 0.0)
    assert d.nb_faces == 18 and np.isclose(d.faces_areas.sum(), mesh_disk(resolution=(3, 6)).faces_areas.sum())
    assert isinstance(mesh_disk(resolution=(3, 6), axial_symmetry=True), RotationSymmetricMesh)
    with pytest.raises(NotImplementedError):
        mesh_disk(axial_symmetry=True, reflection_symmetry=True)
    for max_rad in (0.5, 1.0, 5.0):
        assert mesh_disk(radius=10.0, faces_max_radius=max_rad).faces_radiuses.max() <= max_rad


def test_vertical_cylinder():
    """test_meshes_predefined.py:62-106"""
    v = mesh_vertical_cylinder(resolution=(2, 8, 10), name="foo")
    assert isinstance(v, Mesh) and v.nb_faces == (10 + 2 * 2) * 8 and v.name == "foo"
    v = mesh_vertical_cylinder(center=(-10.0, 5.0, 1.0), length=6.0, radius=4.0, resolution=(0, 100, 5))
    assert np.isclose(np.min(v.vertices[:, 0]), -14.0)
    assert np.isclose(np.min(v.vertices[:, 1]), 1.0)
    assert np.isclose(np.min(v.vertices[:, 2]), -2.0)
    v = mesh_vertical_cylinder(reflection_symmetry=True, center=(0.0, 0.0, 6.0))
    assert isinstance(v, ReflectionSymmetricMesh)
    assert v.merged().nb_faces == mesh_vertical_cylinder(reflection_symmetry=False).nb_faces
    assert np.all(v.half.vertices[:, 0] >= 0.0) and not np.all(v.vertices[:, 0] >= 0.0)
    assert np.all(v.vertices[:, 2] > 0.0)
    assert isinstance(mesh_vertical_cylinder(axial_symmetry=True), RotationSymmetricMesh)
    for max_rad in (0.5, 1.0, 5.0):
        assert mesh_vertical_cylinder(radius=10.0, faces_max_radius=max_rad).faces_radiuses.max() <= max_rad


def test_horizontal_cylinder():
    """test_meshes_predefined.py:108-136"""
    h = mesh_horizontal_cylinder(resolution=(2, 8, 10), name="foo")
    assert isinstance(h, Mesh) and h.nb_faces == (10 + 2 * 2) * 8 and h.name == "foo"
    assert _outward(h)
    h = mesh_horizontal_cylinder(length=10.0, radius=1.0, resolution=(0, 100, 3), center=(10.0, 1.0, 0.0))
    assert np.isclose(np.min(h.vertices[:, 0]), 5.0) and np.isclose(np.min(h.vertices[:, 1]), 0.0)
    h = mesh_horizontal_cylinder(reflection_symmetry=True, center=(0.0, 0.0, 5.0))
    assert isinstance(h, ReflectionSymmetricMesh)
    assert h.merged().nb_faces == mesh_horizontal_cylinder(reflection_symmetry=False).nb_faces
    assert not np.all(h.vertices[:, 1] >= 0.0) and np.all(h.half.vertices[:, 1] >= 0.0)
    assert np.all(h.vertices[:, 2] > 0.0)
    assert _outward(h.merged())
    for max_rad in (0.5, 1.0, 5.0):
        assert mesh_horizontal_cylinder(radius=10.0, faces_max_radius=max_rad).faces_radiuses.max() <= max_rad


def test_sphere():
    """test_meshes_predefined.py:138-168"""
    d = mesh_sphere(resolution=(3, 6), name="foo")
    assert isinstance(d, Mesh) and d.nb_faces == 18 and d.name == "foo"
    d = mesh_sphere(radius=0.1, center=(1.0, 0.5, -0.5))
    assert np.all(d.vertices[:, 0] <= 1.1) and np.all(0.9 <= d.vertices[:, 0])
    assert np.all(d.vertices[:, 2] <= -0.4) and np.all(-0.6 <= d.vertices[:, 2])
    d = mesh_sphere(resolution=(3, 6), axial_symmetry=True)
    assert isinstance(d, RotationSymmetricMesh) and d.axis == "z+"
    for max_rad in (0.5, 1.0, 5.0):
        assert mesh_sphere(radius=10.0, faces_max_radius=max_rad).faces_radiuses.max() <= max_rad
        assert mesh_sphere(radius=10.0, resolution=(10, 10), faces_max_radius=max_rad).faces_radiuses.max() <= max_rad


def test_rectangle():
    """test_meshes_predefined.py:170-208"""
    with pytest.raises(AssertionError):
        mesh_rectangle(size=(-4, 5))
    with pytest.raises(AssertionError):
        mesh_rectangle(resolution=(4.1, 5))
    with pytest.raises(ValueError):
        mesh_rectangle(resolution=(3, 3), reflection_symmetry=True)
    d = mesh_rectangle(resolution=(3, 6), name="foo")
    assert isinstance(d, Mesh) and d.nb_faces == 18 and d.name == "foo"
    d = mesh_rectangle(center=(1.0, 0.5, -0.5), normal=(0, 1, 0))
    assert np.allclose(d.vertices[:, 1], 0.5)
    d = mesh_rectangle(resolution=(4, 6), reflection_symmetry=True, normal=(0, 0, -1))
    assert isinstance(d, ReflectionSymmetricMesh) and np.allclose(d.faces_normals, (0, 0, -1))
    with pytest.raises(ValueError):
        mesh_rectangle(resolution=(4, 6), reflection_symmetry=True, normal=(1, 1, 1))
    for max_rad in (0.5, 1.0, 5.0):
        assert mesh_rectangle(size=(10.0, 10.0), faces_max_radius=max_rad).faces_radiuses.max() <= max_rad


def test_parallelepiped():
    """test_meshes_predefined.py:210-245"""
    p = mesh_parallelepiped(resolution=(3, 6, 3), name="foo")
    assert isinstance(p, Mesh) and p.nb_faces == 90 and p.name == "foo"
    p = mesh_parallelepiped(size=(5.0, 5.0, 5.0), missing_sides=["top", "bottom"])
    assert p.nb_faces == 64
    assert not np.any((abs(p.faces_centers[:, 0]) < 2.0) & (abs(p.faces_centers[:, 1]) < 2.0))
    p = mesh_parallelepiped(center=(2.0, -2.0, 1.0))
    assert np.all(p.faces_centers[:, 0] <= 3.0) and np.all(1.0 <= p.faces_centers[:, 0])
    p = mesh_parallelepiped(resolution=(4, 4, 4), reflection_symmetry=True)
    assert isinstance(p, ReflectionSymmetricMesh) and isinstance(p.half, ReflectionSymmetricMesh)
    assert p.nb_faces == 6 * 16
    for max_rad in (0.5, 1.0, 5.0):
        assert mesh_parallelepiped(size=(10.0, 10.0, 10.0), faces_max_radius=max_rad).faces_radiuses.max() <= max_rad
        assert mesh_parallelepiped(size=(1.0, 10.0, 1.0), faces_max_radius=max_rad).faces_radiuses.max() <= max_rad
