"""Block structure of the influence matrices of a symmetric mesh.

The mesh is the union of the images g_0 h, ..., g_{m-1} h of one sub-mesh h
under a group of symmetries of the free-surface Green function (reflections in
xOz / yOz, rotations about Oz), in capytaine's face order.  The block of the
influence matrices between images I and J depends only on g_I^-1 g_J, so the
first column of blocks C_j = G(g_j h, h) (the whole mesh's collocation points
against the panels of h, capytaine bem/engines.py:178-247) fixes S and K, and
the group's Fourier transform splits the dense system into independent ones
(tools/block_circulant_matrices.py:42-423):

* one plane ("reflection"): m = 2 blocks, systems C_0 + C_1 and C_0 - C_1;
* two planes ("reflections"): m = 4 (group Z2 x Z2, image j = sigma_1^(j & 1)
  sigma_2^(j >> 1) h), 4 systems sum_j (-1)^popcount(k & j) C_j;
* rotation of order n ("rotation"): m = n, n systems sum_j e^(-2 pi i jk/n) C_j;
* rotation of a reflection ("dihedral", order 2n): m = 2n images R^i sigma^s h
  at index 2i + s; macro-blocks of 2 x 2 images are circulant over i, giving n
  systems of twice the sub-mesh size.  Macro-block d (block row I, column
  I - d) is [[C_2d, C_2((n-d) mod n)+1], [C_2d+1, C_2((n-d) mod n)]]: moving
  the image of the column to h by R^-j, or by sigma R^-j when it holds a
  reflection (sigma R^a = R^-a sigma).

For capytaine's two-plane matrices the reference factors two systems of size
N/2 (NestedBlockCirculantMatrix.to_BlockCirculantMatrix, :226-266, then one
circulant split); here the four systems of size N/4 carry the same solution.

Systems k = sum_i W[k, i] M_i with M_i the macro-blocks; a vector v of the
whole mesh (segments v_i of the system size) maps to v^_k = sum_i W[k, i] v_i
and back by v_i = sum_k Winv[i, k] v^_k.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np

from .symmetric_meshes import ReflectionSymmetricMesh, RotationSymmetricMesh


@dataclass(frozen=True, eq=False)
class BlockStructure:
    kind: str              # "reflection", "reflections", "rotation" or "dihedral"
    submesh: object        # plain mesh h: the panels of the first block column
    nb_images: int         # m: images of h in the whole mesh (blocks in the first column)
    q: int                 # images per macro-block side (1, or 2 for dihedral)
    source: np.ndarray     # (nsys, q, q) int32: image block at (macro-block i, row part, column part)
    W: np.ndarray          # (nsys, nsys) complex128
    Winv: np.ndarray       # (nsys, nsys) complex128

    @property
    def nsys(self) -> int:
        return self.W.shape[0]

    @property
    def n_sub(self) -> int:
        return self.submesh.nb_faces

    @property
    def n_sys(self) -> int:
        return self.q * self.n_sub

    def macro_blocks(self, blocks: np.ndarray) -> np.ndarray:
        """(nsys, n_sys, n_sys) macro-blocks from the (m, n_sub, n_sub) first-column blocks."""
        ns = self.n_sub
        out = np.empty((self.nsys, self.n_sys, self.n_sys), dtype=blocks.dtype)
        for i in range(self.nsys):
            for a in range(self.q):
                for b in range(self.q):
                    out[i, a * ns:(a + 1) * ns, b * ns:(b + 1) * ns] = blocks[self.source[i, a, b]]
        return out

    def systems(self, blocks: np.ndarray) -> np.ndarray:
        """(nsys, n_sys, n_sys) independent systems (host reference of the device transform)."""
        return np.einsum("ki,irc->krc", self.W, self.macro_blocks(blocks))

    def full_matrix(self, blocks: np.ndarray) -> np.ndarray:
        """Dense matrix of the whole mesh from the first-column blocks."""
        m, ns = self.nb_images, self.n_sub
        M = np.empty((m * ns, m * ns), dtype=blocks.dtype)
        for I in range(m):
            for J in range(m):
                M[I * ns:(I + 1) * ns, J * ns:(J + 1) * ns] = blocks[self.image_block(I, J)]
        return M

    def image_block(self, I: int, J: int) -> int:
        """Index j of the first-column block equal to block (I, J)."""
        if self.kind == "reflections":
            return I ^ J
        if self.kind == "dihedral":
            n = self.nb_images // 2
            i, s = divmod(I, 2)
            j, t = divmod(J, 2)
            if t == 0:
                return 2 * ((i - j) % n) + s
            return 2 * ((j - i) % n) + (1 - s)
        return (I - J) % self.nb_images


def _cyclic(n: int):
    k = np.arange(n)
    W = np.exp(-2j * np.pi * np.outer(k, k) / n)
    return W, np.conj(W).T / n


def block_structure(mesh) -> Optional[BlockStructure]:
    """The block structure of a mesh with itself, or None for a plain mesh
    (or a symmetry the engines do not use: a reflection of a rotation uses its
    outer reflection only, as capytaine does)."""
    if isinstance(mesh, ReflectionSymmetricMesh):
        half = mesh.half
        if isinstance(half, ReflectionSymmetricMesh) and half.plane != mesh.plane:
            j = np.arange(4)
            W = np.array([[(-1) ** bin(k & i).count("1") for i in j] for k in j], dtype=np.complex128)
            return BlockStructure("reflections", half.half.merged(), 4, 1, j.reshape(4, 1, 1).astype(np.int32),
                                  W, W.T / 4)
        W, Winv = _cyclic(2)
        return BlockStructure("reflection", half.merged(), 2, 1, np.arange(2, dtype=np.int32).reshape(2, 1, 1),
                              W, Winv)
    if isinstance(mesh, RotationSymmetricMesh):
        n = mesh.n
        W, Winv = _cyclic(n)
        if isinstance(mesh.wedge, ReflectionSymmetricMesh):
            src = np.empty((n, 2, 2), dtype=np.int32)
            for d in range(n):
                e = (n - d) % n
                src[d] = [[2 * d, 2 * e + 1], [2 * d + 1, 2 * e]]
            return BlockStructure("dihedral", mesh.wedge.half.merged(), 2 * n, 2, src, W, Winv)
        return BlockStructure("rotation", mesh.wedge.merged(), n, 1, np.arange(n, dtype=np.int32).reshape(n, 1, 1),
                              W, Winv)
    return None
