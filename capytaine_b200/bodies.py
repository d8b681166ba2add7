"""Floating bodies and their rigid-body degrees of freedom.

Restates the parts of capytaine ``bodies/bodies.py`` and ``bodies/dofs.py``
that the frequency solve consumes: dofs as motion fields evaluated at face
centres (``dofs.py:60-98, 139-172``), the hull/lid split of
``mesh_including_lid`` and ``hull_mask`` (``bodies.py:79-111``), and the
per-dof normal components used by the boundary conditions and the pressure
integration (``bodies.py:238-250``).
"""
from __future__ import annotations

from dataclasses import dataclass
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


@dataclass(frozen=True, eq=False)
class DofOnSubmesh:
    """A dof that is zero everywhere except on some faces, where another dof
    defines the motion (capytaine bodies/dofs.py:100-127): the dofs of one body
    inside a joined multibody.  `faces`: boolean mask over the faces of the
    joined hull, whose face centres are the points the motion is evaluated at."""
    dof: object
    faces: np.ndarray

    def evaluate_motion(self, points: np.ndarray) -> np.ndarray:
        motion = np.zeros((points.shape[0], 3))
        motion[self.faces, :] = self.dof.evaluate_motion(points[self.faces, :])
        return motion


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

    def __add__(self, other: "FloatingBody") -> "FloatingBody":
        return join_bodies(self, other)

    def _join_lid(self):
        if "_with_lid" not in self.__dict__:
            if self.lid_mesh is None:
                self.__dict__["_with_lid"] = (self.mesh, np.ones(self.mesh.nb_faces, dtype=bool))
            else:
                # hull.join_meshes(lid) with masks (bodies.py:104-111): for plain meshes
                # the hull faces then the lid faces, vertices concatenated unchanged; a
                # symmetric hull with a lid of the same symmetry stays symmetric (halves
                # or wedges joined), its hull faces in the order of the hull's faces.
                joined, masks = self.mesh.join_meshes(self.lid_mesh, return_masks=True)
                self.__dict__["_with_lid"] = (joined, masks[0])
        return self.__dict__["_with_lid"]

    @property
    def mesh_including_lid(self) -> Mesh:
        return self._join_lid()[0]

    @property
    def hull_mask(self) -> np.ndarray:
        return self._join_lid()[1].copy()

    def dof_normal_components(self) -> np.ndarray:
        """(ndof, N_with_lid): dof(x_i) . n_i on hull faces, 0 on lid faces."""
        mask = self._join_lid()[1]
        out = np.zeros((len(self.dofs), mask.size))
        c, nrm = self.mesh.faces_centers, self.mesh.faces_normals
        for d, dof in enumerate(self.dofs.values()):
            out[d, mask] = np.sum(dof.evaluate_motion(c) * nrm, axis=1)
        return out

    def pressure_weights(self) -> np.ndarray:
        """(ndof, N_with_lid): -(dof . n) area on hull faces (bodies.py:238-250), 0 on lid faces."""
        mask = self._join_lid()[1]
        w = -self.dof_normal_components()
        w[:, mask] *= self.mesh.faces_areas[None, :]
        return w

    def integrate_pressure(self, pressure: np.ndarray) -> Dict[str, complex]:
        """Host version of bodies.py:238-250 on hull pressures (in the order of the hull's faces)."""
        w = self.pressure_weights()[:, self._join_lid()[1]]
        return {name: complex(np.sum(pressure * w[d])) for d, name in enumerate(self.dofs)}


def join_bodies(*bodies, name: Optional[str] = None) -> "FloatingBody":
    """Several bodies as one (capytaine bodies/multibodies.py:34-122): the
    hull meshes joined in order, each dof restricted to the faces of its body
    and named "<body name>__<dof name>" (kept as is when it already holds
    "__"), the lids joined after all hulls."""
    names = [b.name for b in bodies]
    if len(set(names)) < len(names):
        raise ValueError(f"In Multibody, all component bodies must have a distinct name.\nGot: {names}")
    counts = [b.mesh.nb_faces for b in bodies]
    total = sum(counts)
    hull = Mesh(np.concatenate([b.mesh.vertices for b in bodies]),
                [[i + off for i in f] for b, off in zip(bodies, np.cumsum([0] + [b.mesh.nb_vertices
                                                                               for b in bodies[:-1]]))
                 for f in b.mesh._faces], name=name, clean=False)
    dofs = {}
    start = 0
    for b, cnt in zip(bodies, counts):
        mask = np.zeros(total, dtype=bool)
        mask[start:start + cnt] = True
        start += cnt
        for dname, dof in b.dofs.items():
            dofs[dname if "__" in dname else f"{b.name}__{dname}"] = DofOnSubmesh(dof, mask)
    lids = [b.lid_mesh for b in bodies if b.lid_mesh is not None and b.lid_mesh.nb_faces > 0]
    lid = None
    if lids:
        lid = Mesh(np.concatenate([m.vertices for m in lids]),
                   [[i + off for i in f] for m, off in zip(lids, np.cumsum([0] + [m.nb_vertices for m in lids[:-1]]))
                    for f in m._faces], clean=False)
    return FloatingBody(hull, dofs, lid_mesh=lid, name=name or "+".join(names))
