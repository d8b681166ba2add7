"""Host logic of the symmetric engines without a GPU: which mesh pairs share a
block structure (the condition of capytaine bem/engines.py:181-235), the RAM
estimate, and the transform sizes the engine allocates."""
import numpy as np

from capytaine_b200.engine import _shared_structure, _structure_signature, B200Engine
from capytaine_b200.meshes import mesh_parallelepiped, mesh_vertical_cylinder
from capytaine_b200.symmetric_meshes import ReflectionSymmetricMesh, RotationSymmetricMesh
from capytaine_b200.bodies import FloatingBody, rigid_body_dofs


def test_structure_signatures():
    box = mesh_parallelepiped(size=(6, 4, 4), resolution=(4, 4, 4), reflection_symmetry=True).immersed_part()
    cyl = mesh_vertical_cylinder(resolution=(1, 6, 4), axial_symmetry=True).immersed_part()
    assert _structure_signature(box) == ("reflection", "xOz", ("reflection", "yOz", None))
    assert _structure_signature(cyl) == ("rotation", 6, "z+", None)
    assert _structure_signature(box.merged()) is None
    assert _shared_structure(box, box).kind == "reflections"
    assert _shared_structure(cyl, cyl).kind == "rotation"
    assert _shared_structure(box, cyl) is None
    assert _shared_structure(box.merged(), box) is None       # plain collocation mesh
    assert _shared_structure(np.zeros((4, 3)), box) is None  # raw points
    other = ReflectionSymmetricMesh(box.half.half, plane="yOz")
    assert _shared_structure(other, box) is None
    wedge_mesh = RotationSymmetricMesh(cyl.wedge, 6, axis="z-")
    assert _shared_structure(wedge_mesh, cyl) is None        # other orientation


def test_ram_estimation_uses_the_systems():
    class Problem:
        pass
    box = mesh_parallelepiped(size=(80, 20, 20), resolution=(104, 26, 26), reflection_symmetry=True).immersed_part()
    p = Problem()
    p.body = FloatingBody(box, rigid_body_dofs())
    eng = B200Engine.__new__(B200Engine)
    sym = B200Engine.compute_ram_estimation(eng, p)
    p.body = FloatingBody(box.merged(), rigid_body_dofs())
    dense = B200Engine.compute_ram_estimation(eng, p)
    assert 0 < sym < dense / 3
