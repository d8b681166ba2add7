"""Floating bodies and their rigid-body degrees of freedom.

Restates the parts of capytaine ``bodies/bodies.py`` and ``bodies/dofs.py``
that the frequency solve consumes: dofs as motion fields evaluated at face
centres (``dofs.py:60-98, 139-172``), the hull/lid split of
``mesh_including_lid`` and ``hull_mask`` (``bodies.py:79-111``), and the
per-dof normal components used by the boundary conditions and the pressure
integration (``bodies.py:238-250``).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, Optional, Sequence

import numpy as np

from .meshes import Mesh


@dataclass(frozen=True)
class TranslationDof:
    direction: Sequence[float]

    def evaluate_motion(self, points: np.ndarray) -> np.ndarray:
        return np.tile(np.asarray(self.direction, float), (points.shape[0], 1))


@dataclass(frozen=True)
class RotationDof:
    rotation_center: Sequence[float]
    direction: Sequence[float]

    def evaluate_motion(self, points: np.ndarray) -> np.ndarray:
        return np.cross(np.asarray(self.direction, float), points - np.asarray(self.rotation_center, float))


def rigid_body_dofs(only=None, rotation_center=(0.0, 0.0, 0.0)) -> Dict[str, object]:
    """Surge, Sway, Heave, Roll, Pitch, Yaw (capytaine bodies/dofs.py:139-172)."""
    dofs = {
        "Surge": TranslationDof((1, 0, 0)),
        "Sway": TranslationDof((0, 1, 0)),
        "Heave": TranslationDof((0, 0, 1)),
        "Roll": RotationDof(tuple(rotation_center), (1, 0, 0)),
        "Pitch": RotationDof(tuple(rotation_center), (0, 1, 0)),
        "Yaw": RotationDof(tuple(rotation_center), (0, 0, 1)),
    }
    if only is not None:
        dofs = {k: v for k, v in dofs.items() if k in only}
    return dofs


class FloatingBody:
    """A hull mesh, an optional lid mesh (irregular-frequency removal) and dofs."""

    def __init__(self, mesh: Mesh, dofs: Optional[Dict[str, object]] = None, lid_mesh: Optional[Mesh] = None,
                 name: Optional[str] = None):
        self.mesh = mesh
        self.lid_mesh = lid_mesh
        self.dofs = dict(dofs) if dofs is not None else {}
        self.name = name or (mesh.name if mesh.name else "body")

    @property
    def mesh_including_lid(self) -> Mesh:
        if self.lid_mesh is None:
            return self.mesh
        if not hasattr(self, "_with_lid"):
            # Faces of the hull first, then the lid, vertices concatenated (no merge),
            # so face i < nb_hull_faces is hull face i.
            nv = self.mesh.nb_vertices
            faces = [list(f) for f in self.mesh._faces] + [[i + nv for i in f] for f in self.lid_mesh._faces]
            self._with_lid = Mesh(np.concatenate([self.mesh.vertices, self.lid_mesh.vertices]), faces,
                                  quadrature_method=self.mesh.quadrature_method, clean=False)
        return self._with_lid

    @property
    def hull_mask(self) -> np.ndarray:
        n = self.mesh_including_lid.nb_faces
        mask = np.zeros(n, dtype=bool)
        mask[: self.mesh.nb_faces] = True
        return mask

    def dof_normal_components(self) -> np.ndarray:
        """(ndof, N_with_lid): dof(x_i) . n_i on hull faces, 0 on lid faces."""
        n_all = self.mesh_including_lid.nb_faces
        out = np.zeros((len(self.dofs), n_all))
        c, nrm = self.mesh.faces_centers, self.mesh.faces_normals
        for d, dof in enumerate(self.dofs.values()):
            out[d, : self.mesh.nb_faces] = np.sum(dof.evaluate_motion(c) * nrm, axis=1)
        return out

    def pressure_weights(self) -> np.ndarray:
        """(ndof, N_with_lid): -(dof . n) area on hull faces (bodies.py:238-250), 0 on lid faces."""
        w = -self.dof_normal_components()
        w[:, : self.mesh.nb_faces] *= self.mesh.faces_areas[None, :]
        return w

    def integrate_pressure(self, pressure: np.ndarray) -> Dict[str, complex]:
        """Host version of bodies.py:238-250 on hull pressures."""
        w = self.pressure_weights()[:, : self.mesh.nb_faces]
        return {name: complex(np.sum(pressure * w[d])) for d, name in enumerate(self.dofs)}
