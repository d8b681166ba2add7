"""Symmetric meshes and the block structure of their influence matrices, on the
host.  Mesh behaviour follows capytaine's pytest/test_meshes_reflection_symmetry.py
and test_meshes_rotation_symmetry.py (face order, winding, clipping, joins);
the block algebra follows pytest/test_tools_block_circulant_matrices.py (the
block-circulant solve equals the dense solve); the symmetric solve of the
oracle equals its dense solve of the merged mesh, as
pytest/test_bem_solver.py:84-95 asserts for capytaine (rel 1e-4 there; 1e-9 here
for meshes whose faces and images have the same geometry)."""
import numpy as np
import pytest

from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
from capytaine_b200.meshes import Mesh, mesh_parallelepiped, mesh_sphere, mesh_vertical_cylinder
from capytaine_b200.symmetric_meshes import ReflectionSymmetricMesh, RotationSymmetricMesh
from capytaine_b200.symmetry import block_structure


def _square(z=-1.0):
    v = np.array([[0.0, 0.5, z], [1.0, 0.5, z], [1.0, 1.5, z], [0.0, 1.5, z]])
    return Mesh(v, [[0, 1, 2, 3]], clean=False)


def dihedral_cylinder(n=3, per_half=2, nr=1, nz=3, radius=2.0, length=6.0):
    """Vertical cylinder as n wedges, each the mirror pair (in yOz) of a slice
    of angle pi / n: dihedral symmetry of order 2n."""
    half = mesh_vertical_cylinder(length=length, radius=radius, resolution=(nr, per_half, nz), _theta_max=np.pi / n)
    return RotationSymmetricMesh(ReflectionSymmetricMesh(half, plane="yOz"), n)


# ---- meshes -------------------------------------------------------------------
def test_reflection_merged_order_and_winding():
    half = _square()
    for plane, axis in (("xOz", 1), ("yOz", 0)):
        m = ReflectionSymmetricMesh(half, plane=plane)
        assert m.nb_faces == 2
        c = m.faces_centers
        np.testing.assert_allclose(c[1], c[0] * np.where(np.arange(3) == axis, -1, 1))
        # the mirrored face keeps the normal pointing the same way (here -z: both
        # faces are mirror images of a face whose normal is +-z)
        np.testing.assert_allclose(m.faces_normals[1], m.faces_normals[0] * np.where(np.arange(3) == axis, -1, 1))
    with pytest.raises(ValueError):
        ReflectionSymmetricMesh(half, plane="xOy")


def test_nested_planes_order():
    q = _square()
    m = ReflectionSymmetricMesh(ReflectionSymmetricMesh(q, plane="xOz"), plane="yOz")
    c = m.faces_centers
    x, y = c[0, 0], c[0, 1]
    np.testing.assert_allclose(c[:, :2], [[x, y], [x, -y], [-x, y], [-x, -y]])


def test_rotation_merged_order():
    m = RotationSymmetricMesh(_square(), 4)
    c = m.faces_centers
    for i in range(4):
        t = np.pi / 2 * i
        R = np.array([[np.cos(t), -np.sin(t)], [np.sin(t), np.cos(t)]])
        np.testing.assert_allclose(c[i, :2], R @ c[0, :2], atol=1e-14)
    assert RotationSymmetricMesh(_square(), 4, axis="z-").faces_centers[1, 0] > 0  # clockwise
    with pytest.raises(ValueError):
        RotationSymmetricMesh(_square(), 1)


def test_symmetric_generators_match_plain_ones():
    for sym, plain in (
        (mesh_parallelepiped(size=(8, 4, 4), resolution=(8, 4, 4), reflection_symmetry=True),
         mesh_parallelepiped(size=(8, 4, 4), resolution=(8, 4, 4))),
        (mesh_vertical_cylinder(resolution=(2, 12, 4), axial_symmetry=True), mesh_vertical_cylinder(resolution=(2, 12, 4))),
        (mesh_vertical_cylinder(resolution=(2, 12, 4), reflection_symmetry=True),
         mesh_vertical_cylinder(resolution=(2, 12, 4))),
        (mesh_sphere(resolution=(8, 10), axial_symmetry=True), mesh_sphere(resolution=(8, 10))),
    ):
        assert sym.nb_faces == plain.nb_faces
        assert sym.faces_areas.sum() == pytest.approx(plain.faces_areas.sum(), rel=1e-12)
        # same set of face centres (the order follows the symmetry)
        a = np.round(sym.faces_centers, 9)
        b = np.round(plain.faces_centers, 9)
        assert sorted(map(tuple, a)) == sorted(map(tuple, b))
        # outward normals
        assert np.min(np.sum((sym.faces_centers - sym.faces_centers.mean(0)) * sym.faces_normals, axis=1)) > 0
    with pytest.raises(ValueError):
        mesh_parallelepiped(resolution=(3, 4, 4), reflection_symmetry=True)
    with pytest.raises(NotImplementedError):
        mesh_vertical_cylinder(reflection_symmetry=True, axial_symmetry=True)


def test_clipping_keeps_symmetry_for_the_free_surface():
    box = mesh_parallelepiped(size=(8, 4, 4), resolution=(8, 4, 4), reflection_symmetry=True)
    wet = box.immersed_part()
    assert isinstance(wet, ReflectionSymmetricMesh) and isinstance(wet.half, ReflectionSymmetricMesh)
    assert wet.nb_faces == mesh_parallelepiped(size=(8, 4, 4), resolution=(8, 4, 4)).immersed_part().nb_faces
    cyl = mesh_vertical_cylinder(resolution=(2, 12, 4), axial_symmetry=True).immersed_part()
    assert isinstance(cyl, RotationSymmetricMesh)
    # a vertical plane across the symmetry drops it
    cut = box.clipped(origin=(0, 0.5, 0), normal=(0, 1, 0))
    assert isinstance(cut, Mesh)
    # a vertical plane that is its own mirror image keeps it
    kept = ReflectionSymmetricMesh(_square(), plane="xOz").clipped(origin=(0.5, 0, 0), normal=(1, 0, 0))
    assert isinstance(kept, ReflectionSymmetricMesh)


def test_joins_and_lids():
    a = mesh_vertical_cylinder(resolution=(2, 12, 4), reflection_symmetry=True).immersed_part()
    b = ReflectionSymmetricMesh(_square(-0.5), plane="yOz")
    joined, (ma, mb) = a.join_meshes(b, return_masks=True)
    assert isinstance(joined, ReflectionSymmetricMesh)
    np.testing.assert_array_equal(joined.faces_centers[ma], a.faces_centers)
    np.testing.assert_array_equal(joined.faces_centers[mb], b.faces_centers)
    other = ReflectionSymmetricMesh(_square(-0.5), plane="xOz")
    assert isinstance(a.join_meshes(other), Mesh)
    lid = a.generate_lid()
    assert isinstance(lid, ReflectionSymmetricMesh) and lid.nb_faces > 0
    body = FloatingBody(a, rigid_body_dofs(), lid_mesh=lid)
    assert isinstance(body.mesh_including_lid, ReflectionSymmetricMesh)
    mask = body.hull_mask
    assert mask.sum() == a.nb_faces and (~mask).sum() == lid.nb_faces
    np.testing.assert_array_equal(body.mesh_including_lid.faces_centers[mask], a.faces_centers)
    dn = body.dof_normal_components()
    assert np.all(dn[:, ~mask] == 0)
    np.testing.assert_allclose(dn[2, mask], a.faces_normals[:, 2])


# ---- block structure -----------------------------------------------------------
def _symmetric_cases(exact=True):
    """Immersed symmetric meshes of each kind.  exact: open cylinders and a box
    cut at panel edges, whose panels are all rectangles, so each face and its
    image have the same geometry to rounding.  Otherwise the free surface cuts
    panels into triangles and the cylinders have bottom discs: a mirrored
    triangle starts at another vertex, and the face radius (distance from the
    first vertex to the centre, capytaine meshes/geometry.py:80-85) that picks
    exact or one-point Rankine integration differs from the original's, which
    breaks the symmetry of the matrices at the 1e-4 level, in capytaine too
    (its pytest/test_bem_solver.py:84-95 compares at rel 1e-4)."""
    nr, nz = (0, 4) if exact else (1, 3)
    return {
        "reflection": mesh_vertical_cylinder(radius=2.0, length=6.0, resolution=(nr, 8, nz),
                                             reflection_symmetry=True).immersed_part(),
        "reflections": mesh_parallelepiped(size=(6, 4, 4), resolution=(4, 4, nz), reflection_symmetry=True)
        .immersed_part(),
        "rotation": mesh_vertical_cylinder(radius=2.0, length=6.0, resolution=(nr, 6, nz),
                                           axial_symmetry=True).immersed_part(),
        "dihedral": dihedral_cylinder(nr=nr, nz=nz).immersed_part(),
    }


def test_block_structure_kinds():
    cases = _symmetric_cases(exact=False)
    for kind, mesh in cases.items():
        st = block_structure(mesh)
        assert st.kind == kind
        assert st.nb_images * st.n_sub == mesh.nb_faces
        assert st.nsys * st.n_sys == mesh.nb_faces
        np.testing.assert_allclose(st.W @ st.Winv, np.eye(st.nsys), atol=1e-12)
    assert block_structure(mesh_parallelepiped()) is None


@pytest.mark.parametrize("kind", ["reflection", "reflections", "rotation", "dihedral"])
def test_first_block_column_fixes_the_dense_matrices(oracle_mod, legacy_oracle_gf, kind):
    """The dense S and K of the merged mesh equal the matrices rebuilt from the
    first block column, and the independent systems solve the dense system."""
    mesh = _symmetric_cases(exact=True)[kind]
    st = block_structure(mesh)
    full = mesh.merged()
    k = 0.7
    S, K = legacy_oracle_gf.evaluate(full, full, wavenumber=k)
    Sc, Kc = legacy_oracle_gf.evaluate(full, st.submesh, wavenumber=k)
    ns = st.n_sub
    for M, C in ((S, Sc), (K, Kc)):
        blocks = np.ascontiguousarray(C).reshape((st.nb_images, ns, ns))
        rebuilt = st.full_matrix(blocks)
        assert np.abs(rebuilt - M).max() <= 1e-9 * np.abs(M).max()
    blocks = np.ascontiguousarray(Kc).reshape((st.nb_images, ns, ns))
    systems = st.systems(blocks)
    rng = np.random.default_rng(0)
    b = rng.standard_normal(full.nb_faces) + 1j * rng.standard_normal(full.nb_faces)
    bh = np.einsum("ki,ir->kr", st.W, b.reshape(st.nsys, st.n_sys))
    xh = np.stack([np.linalg.solve(systems[j], bh[j]) for j in range(st.nsys)])
    x = np.einsum("ik,kr->ir", st.Winv, xh).reshape(-1)
    ref = np.linalg.solve(K, b)
    assert np.abs(x - ref).max() <= 1e-9 * np.abs(ref).max()


@pytest.mark.parametrize("n,nested", [(2, False), (3, False), (4, False), (10, False), (4, True), (6, True),
                                      (8, True)])
def test_oracle_block_circulant_algebra(oracle_mod, n, nested):
    """Oracle restatement of capytaine's block-circulant classes against dense
    linear algebra and against the group derivation of the package."""
    from capytaine_b200.symmetry import BlockStructure, _cyclic
    rng = np.random.default_rng(n)
    ns = 3
    blocks = rng.standard_normal((n, ns, ns)) + 1j * rng.standard_normal((n, ns, ns))
    blocks[0] += 4 * ns * np.eye(ns)
    macro = oracle_mod.circulant_macro_blocks(blocks, nested)
    nm = len(macro)
    dense = np.block([[macro[(I - J) % nm] for J in range(nm)] for I in range(nm)])
    x = rng.standard_normal(n * ns) + 1j * rng.standard_normal(n * ns)
    np.testing.assert_allclose(oracle_mod.circulant_matvec(macro, x), dense @ x, atol=1e-12)
    sol = oracle_mod.circulant_solve(oracle_mod.circulant_lu(macro), x)
    np.testing.assert_allclose(sol, np.linalg.solve(dense, x), atol=1e-12)
    if nested:  # the package's dihedral / two-plane structure gives the same dense matrix
        if n == 4:
            W = np.array([[(-1) ** bin(k & i).count("1") for i in range(4)] for k in range(4)], dtype=complex)
            st = BlockStructure("reflections", None, 4, 1, np.arange(4, dtype=np.int32).reshape(4, 1, 1), W, W.T / 4)
        else:
            m = n // 2
            src = np.array([[[2 * d, 2 * ((m - d) % m) + 1], [2 * d + 1, 2 * ((m - d) % m)]] for d in range(m)],
                           dtype=np.int32)
            W, Winv = _cyclic(m)
            st = BlockStructure("dihedral", None, n, 2, src, W, Winv)
        mine = np.block([[blocks[st.image_block(I, J)] for J in range(n)] for I in range(n)])
        np.testing.assert_array_equal(mine, dense)


@pytest.mark.parametrize("exact", [True, False])
@pytest.mark.parametrize("kind", ["reflection", "reflections", "rotation", "dihedral"])
def test_oracle_symmetric_solve_equals_dense_solve(oracle_mod, legacy_oracle_gf, kind, exact):
    mesh = _symmetric_cases(exact)[kind]
    st = block_structure(mesh)
    full = mesh.merged()
    dofs = oracle_mod.rigid_body_dofs()
    w = 1.3
    nested = kind in ("reflections", "dihedral")
    sym = oracle_mod.solve_frequency_symmetric(legacy_oracle_gf, full, st.submesh, st.nb_images, nested, dofs, w,
                                               wave_directions=(0.0, 0.6))
    dense = oracle_mod.solve_frequency(legacy_oracle_gf, full, dofs, w, wave_directions=(0.0, 0.6))
    # rounding for exact images; the geometric asymmetry of mirrored triangles otherwise
    tol = 1e-9 if exact else 1e-3
    for fam in ("added_mass", "radiation_damping"):
        a = np.array([[sym[fam][i][j] for j in dofs] for i in dofs])
        b = np.array([[dense[fam][i][j] for j in dofs] for i in dofs])
        assert np.abs(a - b).max() <= tol * np.abs(b).max()
    for beta in (0.0, 0.6):
        a = np.array([sym["excitation"][beta][d] for d in dofs])
        b = np.array([dense["excitation"][beta][d] for d in dofs])
        assert np.abs(a - b).max() <= tol * np.abs(b).max()


# ---- the reference's own mesh tests, on the same panels ---------------------------
def _reflection_panel():
    """pytest/test_meshes_reflection_symmetry.py:29-36"""
    return Mesh(np.array([[0.5, 0.5, 0.0], [1.0, 0.5, 0.0], [1.0, 1.0, 0.0], [0.5, 1.0, 0.0]]), [[0, 1, 2, 3]],
                clean=False)


def _rotation_panel():
    """pytest/test_meshes_rotation_symmetry.py:29-36"""
    return Mesh(np.array([[0.5, 0.0, 0.0], [0.5, 0.0, -0.5], [0.5, 0.5, -0.5], [0.5, 0.5, 0.0]]), [[0, 1, 2, 3]],
                clean=False)


def test_reference_reflection_mesh_cases():
    """test_meshes_reflection_symmetry.py:39-93: sizes, reflected centres, winding."""
    for plane, axis in (("xOz", 1), ("yOz", 0)):
        m = ReflectionSymmetricMesh(_reflection_panel(), plane=plane)
        assert m.plane == plane and m.nb_faces == 2 and m.nb_vertices == 8
        merged = m.merged()
        assert merged.nb_vertices == 8 and merged.nb_faces == 2
        assert np.isclose(merged.faces_centers[0, axis], 0.75) and np.isclose(merged.faces_centers[1, axis], -0.75)
        assert np.isclose(merged.faces_normals[0, 2], 1.0) and np.isclose(merged.faces_normals[1, 2], 1.0)
    nested = ReflectionSymmetricMesh(ReflectionSymmetricMesh(_reflection_panel(), plane="xOz"), plane="yOz")
    assert nested.nb_faces == 4 and nested.nb_vertices == 16
    assert nested.merged().nb_faces == 4 and nested.merged().nb_vertices == 16


def test_reference_clipped_reflection_case():
    """test_meshes_reflection_symmetry.py:248-256: the immersed part of a panel
    crossing the free surface keeps the symmetry and half of the area."""
    half = Mesh(np.array([[0, 0.5, -0.5], [0, 0.5, 0.5], [0, 1.5, 0.5], [0, 1.5, -0.5]]), [[0, 1, 2, 3]],
                clean=False)
    sym = ReflectionSymmetricMesh(half, plane="xOz")
    wet = sym.immersed_part()
    assert isinstance(wet, ReflectionSymmetricMesh)
    assert np.isclose(wet.faces_areas.sum(), 0.5 * sym.faces_areas.sum())


def test_reference_rotation_mesh_cases():
    """test_meshes_rotation_symmetry.py:105-131: a rotation about Oz keeps the
    symmetry, the merged faces are in the mesh's order, and mirroring commutes
    with merging (face order included)."""
    m = RotationSymmetricMesh(_rotation_panel(), 4)
    assert isinstance(m.rotated_z(np.pi / 4), RotationSymmetricMesh)
    np.testing.assert_allclose(m.merged().faces_centers, m.faces_centers)
    np.testing.assert_allclose(m.merged().mirrored("xOz").faces_centers, m.mirrored("xOz").merged().faces_centers,
                               atol=1e-15)
    np.testing.assert_allclose(m.merged().mirrored("yOz").faces_centers, m.mirrored("yOz").merged().faces_centers,
                               atol=1e-15)


@pytest.mark.parametrize("kind", ["reflection", "reflections", "rotation", "dihedral"])
def test_oracle_symmetric_solve_in_finite_depth(oracle_mod, legacy_oracle_gf, kind):
    """The block structure holds in finite depth too (the sea-bottom images and
    the Prony terms are invariant under the same symmetries): the oracle's
    block-circulant solve equals its dense solve at 8 m of water."""
    mesh = _symmetric_cases(True)[kind]
    st = block_structure(mesh)
    full = mesh.merged()
    dofs = oracle_mod.rigid_body_dofs()
    nested = kind in ("reflections", "dihedral")
    sym = oracle_mod.solve_frequency_symmetric(legacy_oracle_gf, full, st.submesh, st.nb_images, nested, dofs, 1.3,
                                               water_depth=8.0)
    dense = oracle_mod.solve_frequency(legacy_oracle_gf, full, dofs, 1.3, water_depth=8.0)
    for fam in ("added_mass", "radiation_damping"):
        a = np.array([[sym[fam][i][j] for j in dofs] for i in dofs])
        b = np.array([[dense[fam][i][j] for j in dofs] for i in dofs])
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()
    a = np.array([sym["excitation"][0.0][d] for d in dofs])
    b = np.array([dense["excitation"][0.0][d] for d in dofs])
    assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()
