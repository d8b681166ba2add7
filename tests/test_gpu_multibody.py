"""Joined bodies with interior lids (irregular-frequency removal) and more
right-hand sides than one solve call takes (12 dofs + 5 headings = 17 columns,
solved in chunks of 16), against the oracle with the same hull mask and
submesh dofs."""
import numpy as np
import pytest

from capytaine_b200.bodies import FloatingBody, join_bodies, rigid_body_dofs
from capytaine_b200.meshes import mesh_vertical_cylinder

pytestmark = pytest.mark.gpu


def _array(oracle_mod):
    bodies, odofs = [], {}
    centers = [(0.0, 0.0), (12.0, 0.0)]
    for i, (x, y) in enumerate(centers):
        h = mesh_vertical_cylinder(length=8.0, radius=2.5, resolution=(3, 24, 8), center=(x, y, 0)).immersed_part()
        bodies.append(FloatingBody(h, rigid_body_dofs(rotation_center=(x, y, 0)), lid_mesh=h.generate_lid(),
                                   name=f"cyl{i}"))
    body = join_bodies(*bodies)
    starts = np.cumsum([0] + [b.mesh.nb_faces for b in bodies])
    for i, (x, y) in enumerate(centers):
        mask = np.zeros(body.mesh.nb_faces, bool)
        mask[starts[i]:starts[i + 1]] = True
        for name, d in oracle_mod.rigid_body_dofs(rotation_center=(x, y, 0)).items():
            odofs[f"cyl{i}__{name}"] = oracle_mod.SubmeshDof(d, mask)
    return body, odofs


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_two_cylinders_with_lids_against_oracle(oracle_mod, default_oracle_gf, tmp_path, precision):
    from capytaine_b200.engine import B200Engine
    from test_gpu_mixed import _shared_table_gf
    from test_gpu_solve import coefficient_errors
    body, odofs = _array(oracle_mod)
    mesh = body.mesh_including_lid
    assert body.lid_mesh.nb_faces > 0 and len(body.dofs) == 12
    heads = (0.0, np.pi / 5, np.pi / 3, np.pi / 2, np.pi)
    omegas = [0.8, 2.1]
    gf = _shared_table_gf(default_oracle_gf, tmp_path)
    res = B200Engine(green_function=gf, precision=precision, max_batch=2).solve_frequencies(
        body, omegas, wave_directions=heads)
    assert res.excitation.shape == (2, len(heads), 12)
    ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh, odofs, w, wave_directions=heads,
                                      hull_mask=body.hull_mask) for w in omegas]
    errs = coefficient_errors(res, ref, body.dofs)
    assert max(errs.values()) < (1e-6 if precision == "fp64" else 1e-5), errs


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_many_bodies_batched_across_bodies(default_oracle_gf, tmp_path, precision):
    """solve_bodies (bodies of uneven sizes sharing identity-padded batches,
    different dof counts) gives each body what solve_frequencies gives it."""
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.meshes import mesh_ellipsoid, mesh_sphere
    from test_gpu_mixed import _shared_table_gf
    gf = _shared_table_gf(default_oracle_gf, tmp_path)
    bodies = [
        FloatingBody(mesh_sphere(radius=1.0, resolution=(10, 20)).immersed_part(), rigid_body_dofs(), name="a"),
        FloatingBody(mesh_ellipsoid(semi_axes=(2.0, 1.0, 1.5), resolution=(10, 22)).immersed_part(),
                     rigid_body_dofs(only=["Heave", "Pitch"]), name="b"),
        FloatingBody(mesh_vertical_cylinder(length=6.0, radius=1.5, resolution=(3, 20, 10)).immersed_part(),
                     rigid_body_dofs(only=["Surge", "Heave", "Yaw"]), name="c"),
    ]
    omegas = [0.5, 1.4, 2.9]
    eng = B200Engine(green_function=gf, precision=precision)
    together = eng.solve_bodies(bodies, omegas, wave_directions=(0.0, np.pi / 4), batch_bytes=3e8)
    assert together[0].stats["groups"] >= 2
    tol = 1e-10 if precision == "fp64" else 1e-8
    for b, res in zip(bodies, together):
        alone = eng.solve_frequencies(b, omegas, wave_directions=(0.0, np.pi / 4))
        for name in ("added_mass", "radiation_damping", "excitation"):
            a, s = getattr(res, name), getattr(alone, name)
            assert a.shape == s.shape
            assert np.abs(a - s).max() <= tol * np.abs(s).max(), (b.name, name)
