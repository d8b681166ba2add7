"""Whole sweeps and the larger configurations against the oracle.

* The 6084-panel barge (80 x 20 m, draft 10 m, 6 rigid dofs about the origin
  + diffraction at heading 0) over every one of the 60 frequencies of its
  linspace(0.05, 3, 60) sweep, for the float64 engine (gate 1e-6) and the
  refined mixed engine (gate 1e-5).  Above 1.3 rad/s the sweep crosses the
  barge's irregular frequencies (the first interior eigenvalue of the box,
  k = kappa coth(kappa T) with kappa = pi sqrt(1/80^2 + 1/20^2) and T = 10 m,
  is at omega = 1.31 rad/s, and they crowd together above it), where K is
  close to singular and the refinement is stressed; the worst frequency of
  each engine is printed.
* Four of the 64 seeded bodies of the many-bodies configuration (ellipsoids
  and vertical cylinders of 300-3000 panels, seed 0, 6 dofs) at 3 of its 30
  frequencies, batched across bodies by solve_bodies, both engines.
* The 3 x 3 array of vertical cylinders (radius 5 m, draft 20 m, spacing
  30 m) with interior lids, about 20000 panels, 54 dofs + diffraction, at 2 of
  its 40 frequencies, refined mixed engine.

The per-coefficient error is the one of the measurement: |c - c_ref| /
max(|c_ref|, 1e-3 max |C_ref|) per family (added mass, damping, excitation),
the floor against couplings that vanish by symmetry."""
import numpy as np
import pytest

from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
from capytaine_b200.meshes import mesh_parallelepiped

pytestmark = pytest.mark.gpu

BARGE_OMEGAS = np.linspace(0.05, 3.0, 60)


def per_omega_errors(res, ref_list, dofs):
    """Worst relative error of each frequency over the three families."""
    from test_gpu_solve import coefficient_errors
    out = []
    for i, ref in enumerate(ref_list):
        one = type(res)(omegas=res.omegas[i:i + 1], dofs=res.dofs, wave_directions=res.wave_directions,
                        added_mass=res.added_mass[i:i + 1], radiation_damping=res.radiation_damping[i:i + 1],
                        diffraction=res.diffraction[i:i + 1], froude_krylov=res.froude_krylov[i:i + 1],
                        excitation=res.excitation[i:i + 1])
        out.append(max(coefficient_errors(one, [ref], dofs).values()))
    return np.array(out)


@pytest.fixture(scope="module")
def barge():
    mesh = mesh_parallelepiped(size=(80, 20, 20), resolution=(104, 26, 26)).immersed_part()
    assert mesh.nb_faces == 6084
    return FloatingBody(mesh, rigid_body_dofs(), name="barge")


@pytest.fixture(scope="module")
def barge_oracle(oracle_mod, default_oracle_gf, barge):
    """The oracle's frequency-solve at each of the 60 frequencies (about 1.5 s
    each on 16 host cores)."""
    odofs = oracle_mod.rigid_body_dofs()
    return [oracle_mod.solve_frequency(default_oracle_gf, barge.mesh, odofs, float(w)) for w in BARGE_OMEGAS]


@pytest.mark.parametrize("precision,gate", [("fp64", 1e-6), ("mixed", 1e-5)])
def test_barge_6084_panels_whole_sweep(default_oracle_gf, tmp_path, barge, barge_oracle, precision, gate):
    from capytaine_b200.engine import B200Engine
    from test_gpu_mixed import _shared_table_gf
    eng = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), precision=precision,
                     max_batch=15)
    res = eng.solve_frequencies(barge, BARGE_OMEGAS)
    errs = per_omega_errors(res, barge_oracle, barge.dofs)
    worst = int(np.argmax(errs))
    print(f"\n{precision}: worst omega {BARGE_OMEGAS[worst]:.3f} rad/s, error {errs[worst]:.3e}; "
          f"median {np.median(errs):.3e}; stats {res.stats}")
    assert np.all(np.isfinite(errs))
    assert errs[worst] < gate, (BARGE_OMEGAS[worst], errs.tolist())


@pytest.mark.parametrize("precision,gate", [("fp64", 1e-6), ("mixed", 1e-5)])
def test_seeded_bodies_batched_against_oracle(oracle_mod, default_oracle_gf, tmp_path, precision, gate):
    from bench import seeded_bodies
    from capytaine_b200.engine import B200Engine
    from test_gpu_mixed import _shared_table_gf
    from test_gpu_solve import coefficient_errors
    bodies = seeded_bodies(0, 4, panels=(300, 3000), all_dofs=True)
    omegas = np.linspace(0.1, 4.0, 30)[::10]
    eng = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), precision=precision,
                     max_batch=16)
    results = eng.solve_bodies(bodies, omegas)
    assert results[0].stats["groups"] >= 2  # uneven sizes: several padded groups
    odofs = oracle_mod.rigid_body_dofs()
    worst = {}
    for b, res in zip(bodies, results):
        ref = [oracle_mod.solve_frequency(default_oracle_gf, b.mesh, odofs, float(w)) for w in omegas]
        worst[f"{b.name} ({b.mesh.nb_faces} panels)"] = max(coefficient_errors(res, ref, b.dofs).values())
    print(f"\n{precision}: {worst}")
    assert max(worst.values()) < gate, worst


def test_cylinder_array_with_lids_against_oracle(oracle_mod, default_oracle_gf, tmp_path):
    from bench import cylinder_array_body
    from capytaine_b200.engine import B200Engine
    from test_gpu_mixed import _shared_table_gf
    from test_gpu_solve import coefficient_errors
    body = cylinder_array_body()
    mesh = body.mesh_including_lid
    assert mesh.nb_faces > 19000 and len(body.dofs) == 54 and body.lid_mesh.nb_faces > 0
    omegas = np.linspace(0.1, 2.0, 40)[[0, 20]]
    eng = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), precision="mixed", max_batch=2)
    res = eng.solve_frequencies(body, omegas)
    # oracle dofs: each cylinder's rigid-body motions about its own axis, on its own faces
    odofs = {}
    start = 0
    for i in range(3):
        for j in range(3):
            x, y = 30.0 * (i - 1), 30.0 * (j - 1)
            nf = body.mesh.nb_faces // 9
            mask = np.zeros(body.mesh.nb_faces, bool)
            mask[start:start + nf] = True
            start += nf
            for name, d in oracle_mod.rigid_body_dofs(rotation_center=(x, y, 0.0)).items():
                odofs[f"cyl{3 * i + j}__{name}"] = oracle_mod.SubmeshDof(d, mask)
    assert list(odofs) == list(body.dofs)
    ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh, odofs, float(w), hull_mask=body.hull_mask)
           for w in omegas]
    errs = coefficient_errors(res, ref, body.dofs)
    print(f"\nmixed, {mesh.nb_faces} panels: {errs}; stats {res.stats}")
    assert max(errs.values()) < 1e-5, errs
