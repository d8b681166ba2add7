"""Clipping against the reference's own tests (pytest/test_meshes_clipping.py:20-122)."""
import numpy as np

from capytaine_b200.meshes import Mesh

SQUARE = ([[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1]], [[0, 1, 2, 3]])


def _counts(mesh):
    quads = int(np.sum(mesh._is_quad))
    return mesh.nb_faces - quads, quads  # triangles, quads


def test_clip_above_and_below():
    mesh = Mesh(*SQUARE)
    above = mesh.clipped(origin=np.array([1.5, 0, 1.5]), normal=np.array([0, 0, 1]))
    assert above.nb_faces == 1 and np.array_equal(above.faces, [[0, 1, 2, 3]])
    below = mesh.clipped(origin=np.array([-0.5, 0, -0.5]), normal=np.array([0, 0, 1]))
    assert below.nb_faces == 0 and below.nb_vertices == 0


def test_clip_partial():
    mesh = Mesh(*SQUARE)
    assert _counts(mesh.clipped(origin=np.array([0.5, 0.0, 0.5]), normal=np.array([0, 0, 1]))) == (2, 0)
    mesh = Mesh([[0, 0, 0], [1, 0, 0], [1, 0, 2], [0, 0, 1]], [[0, 1, 2, 3]])
    assert _counts(mesh.clipped(origin=np.array([0.5, 0, 1.2]), normal=np.array([0, 0, 1]))) == (1, 1)


def test_faces_on_the_free_surface():
    mesh = Mesh([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], [[0, 1, 2, 3]])
    assert mesh.immersed_part().nb_faces == 1
    for dz, expected in ((-1e-10, 1), (1e-9, 1), (1e-7, 0)):  # tolerance 1e-8
        assert mesh.translated((0, 0, dz)).immersed_part().nb_faces == expected
