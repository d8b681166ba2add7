"""The two configurations whose numbers the measurement quotes, at their full
sizes, against the oracle: the 800-panel hemisphere (heave radiation and
diffraction at 20 frequencies, float64 engine at the 1e-6 gate and refined
mixed engine at the 1e-5 gate) and the 6084-panel barge (6 dofs and
diffraction at two frequencies of its 0.05-3 rad/s sweep, one either side of
the first irregular frequency near 1.3 rad/s, refined mixed engine)."""
import numpy as np
import pytest

from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
from capytaine_b200.meshes import mesh_parallelepiped, mesh_sphere

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,gate", [("fp64", 1e-6), ("mixed", 1e-5)])
def test_hemisphere_800_panels_20_frequencies(oracle_mod, default_oracle_gf, tmp_path, precision, gate):
    from capytaine_b200.engine import B200Engine
    from test_gpu_mixed import _shared_table_gf
    from test_gpu_solve import coefficient_errors
    mesh = mesh_sphere(radius=1.0, center=(0, 0, 0), resolution=(40, 40)).immersed_part()
    assert mesh.nb_faces == 800
    body = FloatingBody(mesh, rigid_body_dofs(only=["Heave"]))
    omegas = np.linspace(0.1, 5.0, 20)
    res = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), precision=precision,
                     max_batch=10).solve_frequencies(body, omegas)
    ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh, oracle_mod.rigid_body_dofs(only=["Heave"]), w)
           for w in omegas]
    errs = coefficient_errors(res, ref, body.dofs)
    assert max(errs.values()) < gate, errs


def test_barge_6084_panels_two_frequencies(oracle_mod, default_oracle_gf, tmp_path):
    from capytaine_b200.engine import B200Engine
    from test_gpu_mixed import _shared_table_gf
    from test_gpu_solve import coefficient_errors
    mesh = mesh_parallelepiped(size=(80, 20, 20), resolution=(104, 26, 26)).immersed_part()
    assert mesh.nb_faces == 6084
    body = FloatingBody(mesh, rigid_body_dofs())
    omegas = [1.05, 2.5]
    res = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), precision="mixed",
                     max_batch=2).solve_frequencies(body, omegas)
    ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh, oracle_mod.rigid_body_dofs(), w) for w in omegas]
    errs = coefficient_errors(res, ref, body.dofs)
    assert max(errs.values()) < 1e-5, errs


def test_symmetric_barge_6084_panels(oracle_mod, default_oracle_gf, tmp_path):
    """The barge built with its two symmetry planes: 4 systems of 1521 panels
    per frequency, against the oracle's block-circulant solve."""
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.symmetry import block_structure
    from test_gpu_mixed import _shared_table_gf
    from test_gpu_solve import coefficient_errors
    mesh = mesh_parallelepiped(size=(80, 20, 20), resolution=(104, 26, 26), reflection_symmetry=True).immersed_part()
    st = block_structure(mesh)
    assert (mesh.nb_faces, st.kind, st.nsys, st.n_sys) == (6084, "reflections", 4, 1521)
    body = FloatingBody(mesh, rigid_body_dofs())
    omegas = [1.05, 2.5]
    res = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), precision="mixed",
                     max_batch=2).solve_frequencies(body, omegas)
    ref = [oracle_mod.solve_frequency_symmetric(default_oracle_gf, mesh.merged(), st.submesh, 4, True,
                                                oracle_mod.rigid_body_dofs(), w) for w in omegas]
    errs = coefficient_errors(res, ref, body.dofs)
    assert max(errs.values()) < 1e-5, errs
