"""Panel meshes: geometry arrays consumed by the assembly kernels, and the
generators used by the benchmark workloads.

Face geometry restates capytaine ``meshes/geometry.py:35-118`` (normals from
the diagonals of quads, areas and centres from the two triangles (a, b, c) and
(a, c, d), radius = distance from the first vertex to the centre) and
``meshes/meshes.py:454-486`` (triangles stored as quads whose last vertex is
repeated; default quadrature = one point at the centre weighted by the area).
Generators follow ``meshes/predefined/spheres.py:26-66``,
``rectangles.py:26-213`` and ``cylinders.py:108-205``; clipping follows
``meshes/clip.py`` and the cleaning rules of ``meshes/clean.py``.
"""
from __future__ import annotations

import hashlib
from functools import cached_property
from itertools import product
from typing import List, Optional

import numpy as np

__all__ = [
    "Mesh",
    "mesh_sphere",
    "mesh_ellipsoid",
    "mesh_rectangle",
    "mesh_parallelepiped",
    "mesh_vertical_cylinder",
    "mesh_horizontal_cylinder",
    "mesh_disk",
]


def _as_face_lists(faces) -> List[List[int]]:
    out = []
    for f in faces:
        f = [int(v) for v in f]
        if len(f) == 4 and f[2] == f[3]:
            f = f[:3]
        out.append(f)
    return out


class Mesh:
    """A surface mesh of triangles and quadrilaterals.

    Parameters
    ----------
    vertices: array (V, 3)
    faces: sequence of 3- or 4-vertex index lists (0-based); a 4-index face whose
        last two indices are equal is a triangle, as in capytaine.
    quadrature_method: None (one point at the centre) or "Gauss-Legendre 2".
    clean: merge near-duplicate vertices and drop degenerate faces
        (capytaine ``meshes/clean.py``).
    """

    def __init__(self, vertices, faces, *, quadrature_method: Optional[str] = None,
                 name: Optional[str] = None, clean: bool = True):
        self.vertices = np.array(vertices, dtype=np.float64).reshape(-1, 3)
        self._faces = _as_face_lists(faces)
        if clean and len(self._faces) > 0:
            self.vertices, self._faces = _clean_mesh(self.vertices, self._faces)
        elif clean:
            self.vertices = np.empty((0, 3))  # no face, so no used vertex (meshes/clean.py)
        self.quadrature_method = quadrature_method
        self.name = name

    # -- sizes ---------------------------------------------------------------
    @property
    def nb_faces(self) -> int:
        return len(self._faces)

    @property
    def nb_vertices(self) -> int:
        return self.vertices.shape[0]

    def __repr__(self):
        return f"Mesh(nb_faces={self.nb_faces}, nb_vertices={self.nb_vertices}, name={self.name!r})"

    # -- geometry (capytaine meshes/geometry.py:35-85) -------------------------
    @cached_property
    def faces(self) -> np.ndarray:
        """(N, 4) int array, triangles padded by repeating their last vertex."""
        arr = np.array([f if len(f) == 4 else f + [f[-1]] for f in self._faces], dtype=np.int64)
        return arr.reshape(-1, 4)

    @cached_property
    def _is_quad(self) -> np.ndarray:
        f = self.faces
        return f[:, 2] != f[:, 3]

    @cached_property
    def faces_normals(self) -> np.ndarray:
        v, f, q = self.vertices, self.faces, self._is_quad
        ac = v[f[:, 2]] - v[f[:, 0]]
        bd = v[f[:, 3]] - v[f[:, 1]]
        quad_n = np.cross(ac, bd)
        tri_n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
        n = np.where(q[:, None], quad_n, tri_n)
        return n / np.linalg.norm(n, axis=1)[:, None]

    @cached_property
    def _triangle_parts(self):
        v, f = self.vertices, self.faces
        a, b, c, d = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]], v[f[:, 3]]
        area1 = 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1)
        area2 = np.where(self._is_quad, 0.5 * np.linalg.norm(np.cross(c - a, d - a), axis=1), 0.0)
        return a, b, c, d, area1, area2

    @cached_property
    def faces_areas(self) -> np.ndarray:
        _, _, _, _, area1, area2 = self._triangle_parts
        return np.where(self._is_quad, area1 + area2, area1)

    @cached_property
    def faces_centers(self) -> np.ndarray:
        a, b, c, d, area1, area2 = self._triangle_parts
        c1 = (a + b + c) / 3
        c2 = (a + c + d) / 3
        quad_c = (c1 * area1[:, None] + c2 * area2[:, None]) / (area1 + area2)[:, None]
        return np.where(self._is_quad[:, None], quad_c, c1)

    @cached_property
    def faces_radiuses(self) -> np.ndarray:
        return np.linalg.norm(self.faces_centers - self.vertices[self.faces[:, 0]], axis=1)

    @cached_property
    def quadrature_points(self):
        """(points (N, Q, 3), weights (N, Q)); capytaine meshes/meshes.py:472-486."""
        if self.quadrature_method is None:
            return self.faces_centers.reshape((-1, 1, 3)), self.faces_areas.reshape(-1, 1)
        if self.quadrature_method == "Gauss-Legendre 2":
            return _gauss_legendre_2(self.vertices, self.faces)
        raise ValueError(f"Unknown quadrature_method: {self.quadrature_method}")

    @cached_property
    def z_span(self):
        return float(self.vertices[:, 2].min()), float(self.vertices[:, 2].max())

    @cached_property
    def content_hash(self) -> str:
        """Digest of the vertex and face arrays (cache key for device-resident data)."""
        h = hashlib.sha1()
        h.update(np.ascontiguousarray(self.vertices).tobytes())
        h.update(np.ascontiguousarray(self.faces).tobytes())
        h.update(repr(self.quadrature_method).encode())
        return h.hexdigest()

    def __eq__(self, other):
        return isinstance(other, Mesh) and self.content_hash == other.content_hash

    def __hash__(self):
        return hash(self.content_hash)

    # -- transformations ------------------------------------------------------
    def translated(self, shift, name=None) -> "Mesh":
        return Mesh(self.vertices + np.asarray(shift, dtype=float), self._faces,
                    quadrature_method=self.quadrature_method, name=name or self.name, clean=False)

    def scaled(self, factors, name=None) -> "Mesh":
        return Mesh(self.vertices * np.asarray(factors, dtype=float), self._faces,
                    quadrature_method=self.quadrature_method, name=name or self.name, clean=False)

    def with_quadrature(self, quadrature_method) -> "Mesh":
        return Mesh(self.vertices, self._faces, quadrature_method=quadrature_method, name=self.name, clean=False)

    def mirrored(self, plane: str, name=None) -> "Mesh":
        """Image in the plane xOz (y -> -y) or yOz (x -> -x), each face's vertex
        order reversed so that normals stay outward (capytaine meshes.py:554-573)."""
        v = self.vertices.copy()
        if plane == "xOz":
            v[:, 1] *= -1
        elif plane == "yOz":
            v[:, 0] *= -1
        else:
            raise ValueError(f"Unsupported value for plane: {plane}")
        return Mesh(v, [f[::-1] for f in self._faces], quadrature_method=self.quadrature_method,
                    name=name or self.name, clean=False)

    def rotated_z(self, angle, name=None) -> "Mesh":
        """Rotation by `angle` (radians, counterclockwise seen from +z) about Oz."""
        c, s = np.cos(angle), np.sin(angle)
        R = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
        return Mesh(self.vertices @ R.T, self._faces, quadrature_method=self.quadrature_method,
                    name=name or self.name, clean=False)

    def merged(self) -> "Mesh":
        return self

    def clipped(self, *, origin, normal, name=None) -> "Mesh":
        v, f = _clip_faces(self.vertices, self._faces, np.asarray(normal, float), np.asarray(origin, float))
        return Mesh(v, f, quadrature_method=self.quadrature_method, name=name or self.name, clean=True)

    def generate_lid(self, z=0.0, faces_max_radius=None, name=None) -> "Mesh":
        """Mesh of the interior free surface of the body at height z, for the
        removal of irregular frequencies (capytaine meshes/meshes.py:655-737):
        a rectangle slightly larger than the waterplane (panels of the mean
        face radius of the hull below z, normal -z) keeps the faces whose four
        vertices lie inside the hull, a vertex being inside when an odd number
        of hull faces lie under it in the horizontal projection."""
        if name is None and self.name is not None:
            name = f"lid for {self.name}"
        hull = self.clipped(origin=(0.0, 0.0, z), normal=(0.0, 0.0, 1.0))
        if hull.nb_faces == 0:
            return Mesh(np.empty((0, 3)), [], name=name, clean=False)
        v = hull.vertices
        x_span, y_span = np.ptp(v[:, 0]), np.ptp(v[:, 1])
        x_mean = (v[:, 0].max() + v[:, 0].min()) / 2
        y_mean = (v[:, 1].max() + v[:, 1].min()) / 2
        if faces_max_radius is None:
            faces_max_radius = float(np.mean(hull.faces_radiuses))
        size = (max(faces_max_radius / 2, 1.1 * x_span), max(faces_max_radius / 2, 1.1 * y_span))
        cand = mesh_rectangle(size=(size[1], size[0]), faces_max_radius=faces_max_radius,
                              center=(x_mean, y_mean, z), normal=(0.0, 0.0, -1.0), name="candidate_lid_mesh")
        pts = cand.vertices[:, :2]
        hf = hull.vertices[hull.faces, :2]                      # (F, 4, 2)
        edges = hf[:, [1, 2, 3, 0], :] - hf                    # consecutive vertices of each face
        inside = np.zeros(len(pts), dtype=bool)
        for c0 in range(0, len(pts), 256):  # bounded temporaries: (256, F, 4, 2)
            loc = pts[c0:c0 + 256, None, None, :] - hf[None]
            side = loc[..., 0] * edges[..., 1] - loc[..., 1] * edges[..., 0]
            above = np.all(side <= 0, axis=-1) | np.all(side >= 0, axis=-1)
            inside[c0:c0 + 256] = np.sum(above, axis=-1) % 2 == 1
        keep = np.all(inside[cand.faces], axis=1)
        faces = [list(f) for f in cand.faces[keep]]
        if not faces:
            return Mesh(np.empty((0, 3)), [], name=name, clean=False)
        return Mesh(cand.vertices, faces, name=name, clean=True)

    def immersed_part(self, free_surface=0.0) -> "Mesh":
        """Part below z = free_surface; capytaine abstract_meshes.py:383-407 (infinite depth)."""
        if self.z_span[1] <= free_surface:
            return self
        return self.clipped(origin=(0, 0, free_surface), normal=(0, 0, 1))

    def join_meshes(self, *meshes, return_masks=False, name=None):
        """This mesh and `meshes` as one (symmetric meshes are merged first).
        Without masks the vertices are cleaned; with return_masks the faces are
        concatenated unchanged, in order, and the boolean face mask of each
        input is returned as well (capytaine meshes.py:575-640)."""
        meshes = [m.merged() for m in (self,) + meshes]
        verts, faces, off = [], [], 0
        for m in meshes:
            verts.append(m.vertices)
            faces.extend([[i + off for i in f] for f in m._faces])
            off += m.nb_vertices
        if not return_masks:
            return Mesh(np.concatenate(verts), faces, name=name, clean=True)
        joined = Mesh(np.concatenate(verts), faces, quadrature_method=self.quadrature_method, name=name, clean=False)
        counts = np.cumsum([0] + [m.nb_faces for m in meshes])
        masks = []
        for a, b in zip(counts[:-1], counts[1:]):
            mask = np.zeros(joined.nb_faces, dtype=bool)
            mask[a:b] = True
            masks.append(mask)
        return joined, masks


# ---------------------------------------------------------------------------
def _gauss_legendre_2(vertices, faces):
    """capytaine meshes/geometry.py:88-118."""
    s = 1 / np.sqrt(3)
    local_points = np.array([(s, s), (s, -s), (-s, s), (-s, -s)])
    local_weights = np.array([0.25, 0.25, 0.25, 0.25])
    fv = vertices[faces]
    nb_faces = fv.shape[0]
    points = np.empty((nb_faces, 4, 3))
    weights = np.empty((nb_faces, 4))
    for k, (xk, yk) in enumerate(local_points):
        points[:, k, :] = ((1 + xk) * (1 + yk) * fv[:, 0] + (1 + xk) * (1 - yk) * fv[:, 1]
                           + (1 - xk) * (1 - yk) * fv[:, 2] + (1 - xk) * (1 + yk) * fv[:, 3]) / 4
        dxidx = ((1 + yk) * fv[:, 0] + (1 - yk) * fv[:, 1] - (1 - yk) * fv[:, 2] - (1 + yk) * fv[:, 3]) / 4
        dxidy = ((1 + xk) * fv[:, 0] - (1 + xk) * fv[:, 1] - (1 - xk) * fv[:, 2] + (1 - xk) * fv[:, 3]) / 4
        detJ = np.linalg.norm(np.cross(dxidx, dxidy), axis=1)
        weights[:, k] = local_weights[k] * 4 * detJ
    return points, weights


def _clean_mesh(vertices, faces, tol=1e-8, max_iter=5):
    """Merge near-duplicate vertices, drop repeated indices, degenerate, duplicate
    and small faces, and unused vertices (capytaine meshes/clean.py)."""
    from scipy.spatial import cKDTree

    for _ in range(max_iter):
        nv0, nf0 = len(vertices), len(faces)
        # 1) near-duplicate vertices -> smallest index of each group
        tree = cKDTree(vertices)
        groups = tree.query_ball_tree(tree, r=tol)
        rep_new = {}
        new_vertices = []
        mapping = np.empty(len(vertices), dtype=np.int64)
        for i, group in enumerate(groups):
            rep = min(group)
            if rep not in rep_new:
                rep_new[rep] = len(new_vertices)
                new_vertices.append(vertices[rep])
            mapping[i] = rep_new[rep]
        vertices = np.array(new_vertices)
        faces = [[int(mapping[i]) for i in f] for f in faces]
        # 2) repeated indices inside faces
        new_faces = []
        for f in faces:
            seen, uniq = set(), []
            for vi in f:
                if vi not in seen:
                    seen.add(vi)
                    uniq.append(vi)
            if len(uniq) in (3, 4):
                new_faces.append(uniq)
            elif len(uniq) > 4:
                raise ValueError(f"Face with {len(uniq)} unique vertices: only 3 or 4 supported.")
        faces = new_faces
        # 3) duplicate faces
        seen_f, uniq_faces = set(), []
        for f in faces:
            key = tuple(sorted(f))
            if key not in seen_f:
                seen_f.add(key)
                uniq_faces.append(f)
        faces = uniq_faces
        # 4) small faces (a triangle padded with its last vertex adds a zero second half)
        if faces:
            fv = vertices[np.array([f if len(f) == 4 else f + [f[-1]] for f in faces])]
            areas = 0.5 * (np.linalg.norm(np.cross(fv[:, 1] - fv[:, 0], fv[:, 2] - fv[:, 0]), axis=1)
                           + np.linalg.norm(np.cross(fv[:, 2] - fv[:, 0], fv[:, 3] - fv[:, 0]), axis=1))
            faces = [f for f, a in zip(faces, areas) if a > tol]
        # 5) unused vertices
        used = sorted({i for f in faces for i in f})
        remap = {old: new for new, old in enumerate(used)}
        vertices = vertices[used] if used else np.empty((0, 3))
        faces = [[remap[i] for i in f] for f in faces]
        if len(vertices) == nv0 and len(faces) == nf0:
            break
    return vertices, faces


def _clip_faces(vertices, faces, normal, origin, tol=1e-8):
    """Keep the half-space (origin - v)·normal >= -tol; capytaine meshes/clip.py."""
    verts = vertices.astype(float).tolist()
    new_faces = []
    for face in faces:
        pts = np.asarray([verts[i] for i in face], dtype=float)
        s = (origin - pts) @ normal
        keep = [face[i] for i in range(len(face)) if s[i] >= -tol]
        if len(keep) == 0:
            continue
        if len(keep) == len(face):
            new_faces.append(list(face))
            continue
        keep_set = set(keep)
        edges = list(zip(face, face[1:] + face[:1]))
        inters = {}
        for (i, j) in edges:
            if (i in keep_set) ^ (j in keep_set):
                v1, v2 = np.array(verts[i]), np.array(verts[j])
                u = v2 - v1
                denom = float(np.dot(normal, u))
                if abs(denom) < tol:
                    raise ValueError("Segment is parallel to the plane (no unique intersection).")
                t = float(np.dot(normal, origin - v1) / denom)
                t = max(0.0, min(1.0, t))
                inters[(i, j)] = len(verts)
                verts.append((v1 + t * u).tolist())
        boundary = []
        for (i, j) in edges:
            if i in keep_set:
                boundary.append(i)
            if (i, j) in inters:
                boundary.append(inters[(i, j)])
        if len(boundary) == 3:
            new_faces.append(boundary)
        elif len(boundary) == 4:
            new_faces.append([boundary[0], boundary[1], boundary[2]])
            new_faces.append([boundary[0], boundary[2], boundary[3]])
        elif len(boundary) == 5:
            new_faces.append([boundary[0], boundary[1], boundary[2]])
            new_faces.append([boundary[0], boundary[2], boundary[3], boundary[4]])
        else:
            for k in range(1, len(boundary) - 1):
                new_faces.append([boundary[0], boundary[k], boundary[k + 1]])
    return np.asarray(verts, dtype=float), new_faces


# ---------------------------------------------------------------------------
# Generators
def _surface_of_revolution(profile_points, n):
    """Profile (m, 3) in the xOz half plane, sorted by increasing z, swept n times
    around Oz: faces (i, i+m, i+m+1, i+1) per wedge as in capytaine
    symmetric_meshes.py:410-423, wedges concatenated in order of rotation angle."""
    pts = np.asarray(sorted(list(np.asarray(profile_points, float)), key=lambda p: p[2]))
    m = len(pts)
    verts = []
    for j in range(n):
        t = 2 * np.pi * j / n
        c, s = np.cos(t), np.sin(t)
        rot = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
        verts.append(pts @ rot.T)
    verts = np.concatenate(verts)  # ring j occupies rows [j*m, (j+1)*m)
    faces = []
    for j in range(n):
        jn = (j + 1) % n
        for i in range(m - 1):
            faces.append([j * m + i, jn * m + i, jn * m + i + 1, j * m + i + 1])
    return verts, faces


def mesh_sphere(*, radius=1.0, center=(0.0, 0.0, 0.0), resolution=(10, 10), faces_max_radius=None,
                axial_symmetry=False, name=None):
    """Sphere from a meridian of ntheta+1 points swept nphi times (capytaine
    spheres.py:26-66); with axial_symmetry a RotationSymmetricMesh of nphi
    wedges (same faces, in the same order).  When the panels of `resolution`
    are larger than faces_max_radius, ntheta = nphi = ceil(2 pi R / (sqrt(2)
    faces_max_radius))."""
    ntheta, nphi = resolution
    if faces_max_radius is not None:
        perimeter = 2 * np.pi * radius
        if np.hypot(perimeter / ntheta, perimeter / nphi) / 2 > faces_max_radius:
            ntheta = nphi = int(np.ceil(perimeter / (np.sqrt(2) * faces_max_radius)))
    theta = np.linspace(0.0, np.pi, ntheta + 1)
    meridian = radius * np.stack([np.sin(theta), np.zeros_like(theta), -np.cos(theta)], axis=1)
    if axial_symmetry:
        from .symmetric_meshes import RotationSymmetricMesh
        return RotationSymmetricMesh.from_profile_points(meridian, nphi, name=name).translated(center)
    verts, faces = _surface_of_revolution(meridian, nphi)
    return Mesh(verts, faces, name=name).translated(center)


def mesh_ellipsoid(*, semi_axes=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), resolution=(10, 10), name=None) -> Mesh:
    """Unit sphere scaled along each axis (capytaine has no ellipsoid generator)."""
    return mesh_sphere(radius=1.0, resolution=resolution, name=name).scaled(semi_axes).translated(center)


def mesh_rectangle(*, size=(5.0, 5.0), center=(0.0, 0.0, 0.0), resolution=(5, 5), faces_max_radius=None,
                   normal=(0.0, 0.0, 1.0), reflection_symmetry=False, name=None):
    """One-sided rectangle (capytaine rectangles.py:26-100), built directly in the
    plane orthogonal to ``normal`` with panels oriented along ``normal``.  When
    the panels of ``resolution`` are larger than ``faces_max_radius``, the
    resolution becomes ceil(side / (sqrt(2) faces_max_radius)) per side
    (rectangles.py:67-71).  reflection_symmetry: the half y < 0 mirrored in
    xOz (even number of panels across the width; centre and normal in the
    plane y = 0)."""
    assert len(size) == 2 and all(h > 0 for h in size), "mesh_rectangle: size must be two lengths > 0"
    assert len(resolution) == 2 and all(h > 0 for h in resolution), \
        "mesh_rectangle: resolution must be two panel counts > 0"
    assert all(i == int(i) for i in resolution), "mesh_rectangle: panel counts must be whole numbers"
    assert len(center) == 3, "mesh_rectangle: center must have three coordinates"
    width, height = size
    nw, nh = (int(i) for i in resolution)
    if faces_max_radius is not None and np.hypot(width / nw, height / nh) / 2 > faces_max_radius:
        nw = int(np.ceil(width / (np.sqrt(2) * faces_max_radius)))
        nh = int(np.ceil(height / (np.sqrt(2) * faces_max_radius)))
    if reflection_symmetry:
        from .symmetric_meshes import ReflectionSymmetricMesh
        if nw % 2 == 1:
            raise ValueError("mesh_rectangle: a mirrored rectangle needs an even panel count "
                             "across the mirror plane.")
        if not np.isclose(center[1], 0.0) or not np.isclose(normal[1], 0.0):
            raise ValueError("mesh_rectangle: a mirrored rectangle needs its center and its normal "
                             "in the mirror plane y = 0.")
        half = mesh_rectangle(size=(width / 2, height), resolution=(nw // 2, nh), center=(0, -width / 4, 0),
                              normal=normal)
        return ReflectionSymmetricMesh(half, plane="xOz", name=name).translated(center)
    normal = np.asarray(normal, float)
    normal = normal / np.linalg.norm(normal)
    # In-plane axes: the reference builds the panel in x=0 with normal -x, then rotates.
    a = np.array([-1.0, 0.0, 0.0])
    R = _rotation_aligning(a, normal)
    y_range = np.linspace(-width / 2, width / 2, nw + 1)
    z_range = np.linspace(-height / 2, height / 2, nh + 1)
    nodes = np.array(list(product([0.0], y_range, z_range)), dtype=float)
    panels = [(j + i * (nh + 1), j + 1 + i * (nh + 1), j + 1 + (i + 1) * (nh + 1), j + (i + 1) * (nh + 1))
              for (i, j) in product(range(nw), range(nh))]
    nodes = nodes @ R.T
    return Mesh(nodes, panels, name=name, clean=False).translated(center)


def _rotation_aligning(a, b, eps=1e-8):
    """Rotation matrix taking unit vector a onto unit vector b
    (capytaine abstract_meshes.py:129-175)."""
    a = a / np.linalg.norm(a)
    b = b / np.linalg.norm(b)
    v = np.cross(a, b)
    c = float(np.dot(a, b))
    s = float(np.linalg.norm(v))
    if s < eps and c > 0:
        return np.eye(3)
    if s < eps and c < 0:
        axis = np.eye(3)[int(np.argmin(np.abs(a)))]
        v = np.cross(a, axis)
        v = v / np.linalg.norm(v)
        return 2 * np.outer(v, v) - np.eye(3)
    vx = np.array([[0, -v[2], v[1]], [v[2], 0, -v[0]], [-v[1], v[0], 0]])
    return np.eye(3) + vx + vx @ vx * ((1 - c) / s ** 2)


def mesh_parallelepiped(size=(1.0, 1.0, 1.0), center=(0, 0, 0), resolution=(4, 4, 4), faces_max_radius=None,
                        missing_sides=frozenset(), reflection_symmetry=False, name=None):
    """Six rectangles with outward normals (capytaine rectangles.py:103-213).
    With reflection_symmetry: the quarter x < 0, y < 0 (its sides on the planes
    x = 0 and y = 0 left out) mirrored in yOz, then the half in xOz (even
    resolutions along x and y, centre on Oz)."""
    width, thickness, height = size
    nw, nth, nh = resolution
    if faces_max_radius is not None:
        dw, dh, dth = width / nw, height / nh, thickness / nth
        if max(np.hypot(dw, dh), np.hypot(dw, dth), np.hypot(dth, dh)) / 2 > faces_max_radius:
            nw = int(np.ceil(width / (np.sqrt(2) * faces_max_radius)))
            nth = int(np.ceil(thickness / (np.sqrt(2) * faces_max_radius)))
            nh = int(np.ceil(height / (np.sqrt(2) * faces_max_radius)))
    if reflection_symmetry:
        from .symmetric_meshes import ReflectionSymmetricMesh
        if nw % 2 == 1 or nth % 2 == 1:
            raise ValueError("mesh_parallelepiped: the two mirror planes need even panel counts "
                             "along x and y.")
        if not np.isclose(center[0], 0.0) or not np.isclose(center[1], 0.0):
            raise ValueError("mesh_parallelepiped: the two mirror planes need the center "
                             "on the vertical axis (x = y = 0).")
        quarter = mesh_parallelepiped(size=(width / 2, thickness / 2, height), resolution=(nw // 2, nth // 2, nh),
                                      center=(-width / 4, -thickness / 4, 0),
                                      missing_sides=set(missing_sides) | {"right", "back"})
        half = ReflectionSymmetricMesh(quarter, plane="yOz")
        return ReflectionSymmetricMesh(half, plane="xOz", name=name).translated(center)
    sides = []
    if "left" not in missing_sides:
        sides.append(mesh_rectangle(size=(thickness, height), resolution=(nth, nh), center=(-width / 2, 0, 0),
                                    normal=(-1, 0, 0)))
    if "right" not in missing_sides:
        sides.append(mesh_rectangle(size=(thickness, height), resolution=(nth, nh), center=(width / 2, 0, 0),
                                    normal=(1, 0, 0)))
    if "front" not in missing_sides:
        sides.append(mesh_rectangle(size=(width, height), resolution=(nw, nh), center=(0, -thickness / 2, 0),
                                    normal=(0, -1, 0)))
    if "back" not in missing_sides:
        sides.append(mesh_rectangle(size=(width, height), resolution=(nw, nh), center=(0, thickness / 2, 0),
                                    normal=(0, 1, 0)))
    if "top" not in missing_sides:
        sides.append(mesh_rectangle(size=(thickness, width), resolution=(nth, nw), center=(0, 0, height / 2),
                                    normal=(0, 0, 1)))
    if "bottom" not in missing_sides:
        sides.append(mesh_rectangle(size=(thickness, width), resolution=(nth, nw), center=(0, 0, -height / 2),
                                    normal=(0, 0, -1)))
    return Mesh.join_meshes(*sides, name=name).translated(center)


def mesh_vertical_cylinder(*, length=10.0, radius=1.0, center=(0, 0, 0), resolution=(2, 8, 10),
                           faces_max_radius=None, reflection_symmetry=False, axial_symmetry=False, name=None,
                           _theta_max=2 * np.pi):
    """Closed vertical cylinder: bottom disc, lateral surface, top disc
    (capytaine cylinders.py:108-205).  reflection_symmetry: the half
    0 <= theta <= pi mirrored in yOz (even ntheta); axial_symmetry: one slice of
    angle 2 pi / ntheta repeated ntheta times about Oz."""
    assert length > 0 and radius > 0, "cylinder: length and radius must be > 0"
    nr, ntheta, nz = resolution
    nr, ntheta, nz = _cylinder_resolution(length, radius, nr, ntheta, nz, faces_max_radius)
    if reflection_symmetry and axial_symmetry:
        raise NotImplementedError("mesh_vertical_cylinder: reflection and axial symmetry together are not supported")
    if reflection_symmetry or axial_symmetry:
        from .symmetric_meshes import ReflectionSymmetricMesh, RotationSymmetricMesh
        if reflection_symmetry:
            if ntheta % 2 == 1:
                raise ValueError("a mirrored mesh needs an even number of panels "
                                 "around the axis (ntheta).")
            half = mesh_vertical_cylinder(length=length, radius=radius, resolution=(nr, ntheta // 2, nz),
                                          _theta_max=_theta_max / 2)
            mesh = ReflectionSymmetricMesh(half, plane="yOz", name=name)
        else:
            piece = mesh_vertical_cylinder(length=length, radius=radius, resolution=(nr, 1, nz),
                                           _theta_max=_theta_max / ntheta)
            mesh = RotationSymmetricMesh(piece, ntheta, axis="z+", name=name)
        return mesh.translated(center)
    theta_range = np.linspace(0, _theta_max, ntheta + 1)
    z_range = np.linspace(-length / 2, length / 2, nz + 1)
    if nr > 0:
        r_range = np.linspace(0.0, radius, nr + 1)
        nodes = np.concatenate([
            np.array([(r * np.sin(t), r * np.cos(t), -length / 2) for (r, t) in product(r_range, theta_range)]),
            np.array([(radius * np.sin(t), radius * np.cos(t), z) for (z, t) in product(z_range, theta_range)]),
            np.array([(r * np.sin(t), r * np.cos(t), length / 2) for (r, t) in product(r_range[::-1], theta_range)]),
        ])
    else:
        r_range = np.array([])
        nodes = np.array([(radius * np.sin(t), radius * np.cos(t), z) for (z, t) in product(z_range, theta_range)])
    panels = [(j + i * (ntheta + 1), j + (i + 1) * (ntheta + 1), j + 1 + (i + 1) * (ntheta + 1), j + 1 + i * (ntheta + 1))
              for (i, j) in product(range(nz + 2 * len(r_range)), range(ntheta))]
    return Mesh(nodes, panels, name=name, clean=True).translated(center)


def _cylinder_resolution(length, radius, nr, ntheta, nl, faces_max_radius):
    """Resolution of a cylinder whose panels are at most faces_max_radius
    (cylinders.py:148-157, 242-251): ceil(R / (sqrt(2) r)) along a radius,
    2 ceil(pi R / (sqrt(2) r)) around, ceil(L / (sqrt(2) r)) along the axis."""
    if faces_max_radius is None:
        return nr, ntheta, nl
    dr, dtheta, dl = radius / max(nr, 1e-300), 2 * np.pi * radius / ntheta, length / nl
    if max(np.hypot(dr, dtheta), np.hypot(dtheta, dl)) / 2 > faces_max_radius:
        nr = int(np.ceil(radius / (np.sqrt(2) * faces_max_radius)))
        ntheta = 2 * int(np.ceil(np.pi * radius / (np.sqrt(2) * faces_max_radius)))
        nl = int(np.ceil(length / (np.sqrt(2) * faces_max_radius)))
    return nr, ntheta, nl


def _rotated_to(mesh, a, b):
    """The mesh rotated so that vector a points along b (a symmetric mesh keeps
    its symmetry when a is already b; otherwise it is merged first)."""
    a = np.asarray(a, float) / np.linalg.norm(a)
    b = np.asarray(b, float) / np.linalg.norm(b)
    R = _rotation_aligning(a, b)
    if np.allclose(R, np.eye(3), rtol=0, atol=1e-15):
        return mesh
    m = mesh.merged()
    return Mesh(m.vertices @ R.T, m._faces, quadrature_method=m.quadrature_method, name=m.name, clean=False)


def mesh_disk(*, radius=1.0, center=(0.0, 0.0, 0.0), normal=(0.0, 0.0, 1.0), resolution=(3, 6),
              faces_max_radius=None, reflection_symmetry=False, axial_symmetry=False, name=None,
              _theta_max=2 * np.pi):
    """One-sided disk (capytaine cylinders.py:26-105): nr rings of ntheta panels
    (triangles at the centre), built in the plane x = 0 and turned so that
    its normal is `normal`.  reflection_symmetry: the half y >= 0 mirrored in
    xOz (even ntheta); axial_symmetry: one sector repeated ntheta times about
    Oz (for a horizontal disk)."""
    assert radius > 0, "mesh_disk: radius must be > 0"
    assert len(resolution) == 2 and all(h > 0 for h in resolution), \
        "mesh_disk: resolution must be two counts > 0"
    assert all(i == int(i) for i in resolution), "mesh_disk: counts must be whole numbers"
    nr, ntheta = (int(i) for i in resolution)
    if faces_max_radius is not None and np.hypot(radius / nr, 2 * np.pi * radius / ntheta) / 2 > faces_max_radius:
        nr = int(np.ceil(radius / (np.sqrt(2) * faces_max_radius)))
        ntheta = int(np.ceil(2 * np.pi * radius / (np.sqrt(2) * faces_max_radius)))
    if reflection_symmetry and axial_symmetry:
        raise NotImplementedError("mesh_disk: reflection and axial symmetry together are not supported")
    if reflection_symmetry or axial_symmetry:
        from .symmetric_meshes import ReflectionSymmetricMesh, RotationSymmetricMesh
        if reflection_symmetry:
            if ntheta % 2 == 1:
                raise ValueError("a mirrored mesh needs an even number of panels "
                                 "around the axis (ntheta).")
            half = mesh_disk(radius=radius, resolution=(nr, ntheta // 2), _theta_max=_theta_max / 2)
            mesh = ReflectionSymmetricMesh(half, plane="xOz", name=name)
        else:
            piece = mesh_disk(radius=radius, resolution=(nr, 1), _theta_max=_theta_max / ntheta)
            mesh = RotationSymmetricMesh(piece, ntheta, axis="z+", name=name)
    else:
        theta_range = np.linspace(0, _theta_max, ntheta + 1)
        r_range = np.linspace(0.0, radius, nr + 1)
        nodes = np.array([(0.0, r * np.sin(t), -r * np.cos(t)) for (r, t) in product(r_range, theta_range)])
        panels = [(j + i * (ntheta + 1), j + 1 + i * (ntheta + 1), j + 1 + (i + 1) * (ntheta + 1),
                   j + (i + 1) * (ntheta + 1)) for (i, j) in product(range(nr), range(ntheta))]
        mesh = Mesh(nodes, panels, name=name, clean=True)
    mesh = _rotated_to(mesh, mesh.faces_normals[0], normal)
    return mesh.translated(center, name=name)


def mesh_horizontal_cylinder(*, length=10.0, radius=1.0, center=(0.0, 0.0, 0.0), resolution=(2, 8, 10),
                             faces_max_radius=None, reflection_symmetry=False, name=None, _theta_max=2 * np.pi):
    """Closed cylinder along Ox (capytaine cylinders.py:204-288): nx slices of
    ntheta panels, two end disks of nr rings.  reflection_symmetry: the half
    y >= 0 mirrored in xOz (even ntheta)."""
    assert length > 0 and radius > 0, "cylinder: length and radius must be > 0"
    assert len(resolution) == 3 and all(h >= 0 for h in resolution), \
        "mesh_horizontal_cylinder: resolution must be three counts >= 0"
    nr, ntheta, nx = _cylinder_resolution(length, radius, *(int(i) for i in resolution), faces_max_radius)
    if reflection_symmetry:
        from .symmetric_meshes import ReflectionSymmetricMesh
        if ntheta % 2 == 1:
            raise ValueError("a mirrored mesh needs an even number of panels "
                             "around the axis (ntheta).")
        half = mesh_horizontal_cylinder(length=length, radius=radius, resolution=(nr, ntheta // 2, nx),
                                        _theta_max=_theta_max / 2)
        return ReflectionSymmetricMesh(half, plane="xOz", name=name).translated(center, name=name)
    theta_range = np.linspace(0, _theta_max, ntheta + 1)
    x_range = np.linspace(-length / 2, length / 2, nx + 1)
    nodes = np.array([(x, radius * np.sin(t), -radius * np.cos(t)) for (x, t) in product(x_range, theta_range)])
    panels = [(i + j * (ntheta + 1), i + 1 + j * (ntheta + 1), i + 1 + (j + 1) * (ntheta + 1),
               i + (j + 1) * (ntheta + 1)) for (i, j) in product(range(ntheta), range(nx))]
    mesh = Mesh(nodes, panels, name=name, clean=True)
    if nr > 0:
        side = mesh_disk(radius=radius, center=(-length / 2, 0, 0), normal=(-1, 0, 0), resolution=(nr, ntheta),
                         _theta_max=_theta_max)
        mesh = mesh.join_meshes(side, side.mirrored("yOz"), name=name)
    return mesh.translated(center, name=name)
