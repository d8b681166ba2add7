"""Meshes with reflection or rotation symmetry (capytaine
``meshes/symmetric_meshes.py``).

A ``ReflectionSymmetricMesh`` stores half of a mesh and the plane (xOz or yOz)
that reflects it onto the other half; a ``RotationSymmetricMesh`` stores one
wedge and the order n of the rotation about Oz.  They nest: a reflection of a
reflection (two planes), or a rotation of a reflection (dihedral symmetry).
The face order of the whole mesh is the one capytaine uses: the first half then
the mirrored half, or the wedges in order of rotation angle, recursively.  Every
array a solver reads (vertices, faces, centres, normals, areas, radii,
quadrature points) is the one of that whole (merged) mesh, so a symmetric mesh
goes wherever a plain mesh does; ``B200Engine.solve_frequencies`` also reads
the symmetry and solves the block-diagonalised systems instead
(``capytaine_b200.symmetry``).
"""
from __future__ import annotations

from functools import cached_property
from typing import Optional

import numpy as np

from .meshes import Mesh

__all__ = ["ReflectionSymmetricMesh", "RotationSymmetricMesh"]

_MIRRORED_AXIS = {"xOz": 1, "yOz": 0}


class _SymmetricMesh:
    """Arrays of the merged mesh, shared by both kinds of symmetry."""

    name: Optional[str] = None

    def _build_merged(self) -> Mesh:
        raise NotImplementedError

    def merged(self) -> Mesh:
        if "_merged" not in self.__dict__:
            self.__dict__["_merged"] = self._build_merged()
        return self.__dict__["_merged"]

    @property
    def nb_faces(self) -> int:
        return self.merged().nb_faces

    @property
    def nb_vertices(self) -> int:
        return self.merged().nb_vertices

    @property
    def vertices(self) -> np.ndarray:
        return self.merged().vertices

    @property
    def _faces(self):
        return self.merged()._faces

    @property
    def faces(self) -> np.ndarray:
        return self.merged().faces

    @property
    def faces_normals(self) -> np.ndarray:
        return self.merged().faces_normals

    @property
    def faces_areas(self) -> np.ndarray:
        return self.merged().faces_areas

    @property
    def faces_centers(self) -> np.ndarray:
        return self.merged().faces_centers

    @property
    def faces_radiuses(self) -> np.ndarray:
        return self.merged().faces_radiuses

    @property
    def quadrature_points(self):
        return self.merged().quadrature_points

    @property
    def quadrature_method(self):
        return self.merged().quadrature_method

    @property
    def z_span(self):
        return self.merged().z_span

    @cached_property
    def content_hash(self) -> str:
        return self.merged().content_hash

    def __eq__(self, other):
        return type(other) is type(self) and self.content_hash == other.content_hash

    def __hash__(self):
        return hash((type(self).__name__, self.content_hash))

    def immersed_part(self, free_surface=0.0):
        if self.z_span[1] <= free_surface:
            return self
        return self.clipped(origin=(0.0, 0.0, free_surface), normal=(0.0, 0.0, 1.0))


class ReflectionSymmetricMesh(_SymmetricMesh):
    """`half` and its mirror image in `plane` ("xOz": y -> -y, "yOz": x -> -x);
    faces of the whole mesh: those of `half`, then those of the mirror image
    (capytaine symmetric_meshes.py:30-311)."""

    def __init__(self, half, *, plane: str, name: Optional[str] = None):
        if plane not in _MIRRORED_AXIS:
            raise ValueError(f"Plane must be 'xOz' or 'yOz', got '{plane}'")
        self.half = half
        self.plane = plane
        self.other_half = half.mirrored(plane) if half.nb_faces > 0 else half
        self.name = str(name) if name is not None else None

    def __repr__(self):
        return f"ReflectionSymmetricMesh(half={self.half!r}, plane={self.plane!r}, name={self.name!r})"

    def _build_merged(self) -> Mesh:
        joined, _ = self.half.merged().join_meshes(self.other_half.merged(), return_masks=True, name=self.name)
        return joined

    def _keeps(self, vector) -> bool:
        return abs(float(vector[_MIRRORED_AXIS[self.plane]])) < 1e-12

    def mirrored(self, plane: str, name=None) -> "ReflectionSymmetricMesh":
        return ReflectionSymmetricMesh(self.half.mirrored(plane), plane=self.plane, name=name)

    def rotated_z(self, angle, name=None) -> Mesh:
        return self.merged().rotated_z(angle, name=name)

    def translated(self, shift, name=None):
        if self._keeps(shift):
            return ReflectionSymmetricMesh(self.half.translated(shift), plane=self.plane, name=name or self.name)
        return self.merged().translated(shift, name=name)

    def with_quadrature(self, quadrature_method) -> "ReflectionSymmetricMesh":
        return ReflectionSymmetricMesh(self.half.with_quadrature(quadrature_method), plane=self.plane, name=self.name)

    def clipped(self, *, origin, normal, name=None):
        """Keeps the symmetry when the plane is its own mirror image (normal
        orthogonal to the mirrored axis), as the free surface is."""
        if self._keeps(normal):
            return ReflectionSymmetricMesh(self.half.clipped(origin=origin, normal=normal), plane=self.plane,
                                           name=name or self.name)
        return self.merged().clipped(origin=origin, normal=normal, name=name)

    def generate_lid(self, z=0.0, faces_max_radius=None, name=None) -> "ReflectionSymmetricMesh":
        return ReflectionSymmetricMesh(self.half.generate_lid(z=z, faces_max_radius=faces_max_radius),
                                       plane=self.plane, name=name)

    def join_meshes(self, *meshes, return_masks=False, name=None):
        """Halves joined when every mesh has this symmetry (the mask of each
        input is its half mask twice), else the merged meshes joined."""
        if all(isinstance(m, ReflectionSymmetricMesh) and m.plane == self.plane for m in meshes):
            half, half_masks = self.half.join_meshes(*[m.half for m in meshes], return_masks=True)
            joined = ReflectionSymmetricMesh(half, plane=self.plane, name=name)
            if return_masks:
                return joined, [np.concatenate([hm, hm]) for hm in half_masks]
            return joined
        return self.merged().join_meshes(*[m.merged() for m in meshes], return_masks=return_masks, name=name)


class RotationSymmetricMesh(_SymmetricMesh):
    """`wedge` and its n - 1 images by the rotations of 2 pi i / n about Oz
    (counterclockwise seen from +z for axis "z+", clockwise for "z-"); faces of
    the whole mesh: wedge after wedge (capytaine symmetric_meshes.py:314-662)."""

    def __init__(self, wedge, n: int, *, axis: str = "z+", name: Optional[str] = None):
        if n < 2:
            raise ValueError(f"Rotation order must be >= 2, got: {n}")
        if axis not in ("z+", "z-"):
            raise ValueError(f"Unsupported axis for RotationSymmetricMesh: {axis}")
        self.wedge = wedge
        self.n = int(n)
        self.axis = axis
        sign = 1.0 if axis == "z+" else -1.0
        self.all_wedges = [wedge] + [wedge.rotated_z(sign * 2 * np.pi * i / n) for i in range(1, n)]
        self.name = str(name) if name is not None else None

    def __repr__(self):
        return f"RotationSymmetricMesh(wedge={self.wedge!r}, n={self.n}, axis={self.axis!r}, name={self.name!r})"

    @classmethod
    def from_profile_points(cls, points, n: int, *, name=None) -> "RotationSymmetricMesh":
        """The profile `points` (sorted by increasing z, so that normals point
        outward) swept n times about Oz; the wedge holds the faces between the
        profile and its first rotated copy (symmetric_meshes.py:386-423)."""
        c, s = np.cos(2 * np.pi / n), np.sin(2 * np.pi / n)
        R = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
        pts = np.asarray(sorted(list(np.asarray(points, dtype=float)), key=lambda p: p[2]))
        m = len(pts)
        wedge = Mesh(np.concatenate([pts, pts @ R.T]), [[i, i + m, i + m + 1, i + 1] for i in range(m - 1)])
        return cls(wedge, n, name=name)

    def _build_merged(self) -> Mesh:
        first, *rest = [w.merged() for w in self.all_wedges]
        joined, _ = first.join_meshes(*rest, return_masks=True, name=self.name)
        return joined

    def _opposite_axis(self):
        return "z-" if self.axis == "z+" else "z+"

    def mirrored(self, plane: str, name=None) -> "RotationSymmetricMesh":
        return RotationSymmetricMesh(self.wedge.mirrored(plane), self.n, axis=self._opposite_axis(), name=name)

    def rotated_z(self, angle, name=None) -> "RotationSymmetricMesh":
        return RotationSymmetricMesh(self.wedge.rotated_z(angle), self.n, axis=self.axis, name=name or self.name)

    def translated(self, shift, name=None):
        if abs(float(shift[0])) < 1e-12 and abs(float(shift[1])) < 1e-12:
            return RotationSymmetricMesh(self.wedge.translated(shift), self.n, axis=self.axis, name=name or self.name)
        return self.merged().translated(shift, name=name)

    def with_quadrature(self, quadrature_method) -> "RotationSymmetricMesh":
        return RotationSymmetricMesh(self.wedge.with_quadrature(quadrature_method), self.n, axis=self.axis,
                                     name=self.name)

    def clipped(self, *, origin, normal, name=None):
        """Keeps the symmetry for horizontal planes."""
        if abs(float(normal[0])) < 1e-12 and abs(float(normal[1])) < 1e-12:
            return RotationSymmetricMesh(self.wedge.clipped(origin=origin, normal=normal), self.n, axis=self.axis,
                                         name=name or self.name)
        return self.merged().clipped(origin=origin, normal=normal, name=name)

    def generate_lid(self, z=0.0, faces_max_radius=None, name=None) -> "RotationSymmetricMesh":
        return RotationSymmetricMesh(self.wedge.generate_lid(z=z, faces_max_radius=faces_max_radius), self.n,
                                     axis=self.axis, name=name)

    def join_meshes(self, *meshes, return_masks=False, name=None):
        """Wedges joined when every mesh has this symmetry (the mask of each
        input is its wedge mask n times), else the merged meshes joined."""
        if all(isinstance(m, RotationSymmetricMesh) and m.n == self.n and m.axis == self.axis for m in meshes):
            wedge, wedge_masks = self.wedge.join_meshes(*[m.wedge for m in meshes], return_masks=True)
            joined = RotationSymmetricMesh(wedge, self.n, axis=self.axis, name=name)
            if return_masks:
                return joined, [np.concatenate([wm] * self.n) for wm in wedge_masks]
            return joined
        return self.merged().join_meshes(*[m.merged() for m in meshes], return_masks=return_masks, name=name)
