"""Finite depth and limit frequencies on the device against the CPU oracle,
beyond the assembly parity of test_gpu_assembly_finite_depth.py: complex64
outputs and gradient planes of the finite-depth kernel, finite-depth solves of
B200Engine.solve_frequencies (dense and symmetric meshes, float64 and mixed
engines, finite-depth Airy right-hand sides) at the gates of the
frequency-solve metric, and omega = 0 and infinity inside frequency sweeps
against the oracle's symbolic-frequency radiation solve.  The file name sorts
after every other test file, so that these newer cases run after the rest of
the device suite."""
import dataclasses

import numpy as np
import pytest

from capytaine_b200.meshes import mesh_sphere
from test_gpu_assembly_finite_depth import _close, _gpu_gf, _hemisphere

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("depth,k,sing,kw", [
    (5.0, 1.0, "low_freq", dict(early_dot_product=False)),
    (3.0, 0.7, "high_freq", dict(early_dot_product=False, adjoint_double_layer=False)),
])
def test_finite_depth_gradient_planes(oracle_mod, default_oracle_gf, tmp_path, depth, k, sing, kw):
    """The three gradient planes (early_dot_product=False), for K and for D."""
    mesh = _hemisphere()
    ora = oracle_mod.OracleDelhommeau(gf_singularities=sing, tabulation=default_oracle_gf.tabulation)
    gf = _gpu_gf(default_oracle_gf, tmp_path, gf_singularities=sing)
    decomposition = gf.find_best_exponential_decomposition(k * depth)
    S_ref, K_ref = ora.evaluate(mesh, mesh, wavenumber=k, water_depth=depth, prony=decomposition, **kw)
    S, K = gf.evaluate(mesh, mesh, wavenumber=k, water_depth=depth, **kw)
    assert K.shape == (3, mesh.nb_faces, mesh.nb_faces)
    _close(S, S_ref, 1e-10)
    _close(K, K_ref, 1e-10)


def test_finite_depth_complex64_outputs(oracle_mod, default_oracle_gf, tmp_path):
    """floating_point_precision="float32": complex64 outputs of the same
    float64 arithmetic, within float32 rounding of the oracle's entries."""
    mesh = _hemisphere()
    depth, k = 4.0, 1.3
    gf = _gpu_gf(default_oracle_gf, tmp_path, floating_point_precision="float32")
    decomposition = gf.find_best_exponential_decomposition(k * depth)
    for kw in ({}, dict(early_dot_product=False)):
        S_ref, K_ref = default_oracle_gf.evaluate(mesh, mesh, wavenumber=k, water_depth=depth,
                                                  prony=decomposition, **kw)
        S, K = gf.evaluate(mesh, mesh, wavenumber=k, water_depth=depth, **kw)
        assert S.dtype == np.complex64 and K.dtype == np.complex64
        _close(S, S_ref, 1e-6)
        _close(K, K_ref, 1e-6)


@pytest.mark.parametrize("precision,gate", [("fp64", 1e-6), ("mixed", 1e-5)])
def test_finite_depth_frequency_solve_matches_oracle(oracle_mod, default_oracle_gf, tmp_path, precision, gate):
    """B200Engine.solve_frequencies(water_depth=h): wavenumbers of the
    finite-depth dispersion relation, the finite-depth assembly, the LU, the
    finite-depth Airy right-hand sides and Froude-Krylov forces, against the
    oracle's finite-depth solve; a shallow case (Airy profiles cosh / sinh) and
    a deep one where k h >= 20 at the highest frequency (profiles e^{kz}).
    Gates of the frequency-solve metric (float64 1e-6, mixed 1e-5 per
    coefficient, floor 1e-3 of the largest): the float64 solve was seen at
    4.7e-8 in 50 m of water (a few 1e-11 of the largest coefficient)."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    from test_gpu_solve import coefficient_errors
    mesh = mesh_sphere(radius=1.0, resolution=(10, 20)).immersed_part()
    body = FloatingBody(mesh, rigid_body_dofs())
    heads = (0.0, np.pi / 3)
    eng = B200Engine(green_function=_gpu_gf(default_oracle_gf, tmp_path), precision=precision, max_batch=2)
    odofs = oracle_mod.rigid_body_dofs()
    for depth, omegas in ((3.0, np.array([0.6, 1.4, 3.0])), (50.0, np.array([0.6, 3.0]))):
        res = eng.solve_frequencies(body, omegas, wave_directions=heads, water_depth=depth)
        ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh, odofs, w, wave_directions=heads,
                                          water_depth=depth) for w in omegas]
        errs = coefficient_errors(res, ref, body.dofs)
        assert max(errs.values()) < gate, (depth, errs)


@pytest.mark.parametrize("kind", ["reflections", "rotation"])
def test_finite_depth_symmetric_frequency_solve_matches_oracle(oracle_mod, default_oracle_gf, tmp_path, kind):
    """Meshes with symmetries in finite depth: the first block column assembled
    by the finite-depth kernel (the whole mesh's points against the sub-mesh),
    the block-diagonalised systems, against the oracle's block-circulant solve
    in the same depth."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.symmetry import block_structure
    from test_gpu_solve import coefficient_errors
    from test_symmetry_cpu import _symmetric_cases
    mesh = _symmetric_cases(exact=False)[kind]
    body = FloatingBody(mesh, rigid_body_dofs())
    depth, omegas, heads = 5.0, np.array([0.7, 1.8]), (0.0, 0.7)
    eng = B200Engine(green_function=_gpu_gf(default_oracle_gf, tmp_path), max_batch=2)
    res = eng.solve_frequencies(body, omegas, wave_directions=heads, water_depth=depth)
    assert res.stats["symmetry"] == kind
    st = block_structure(mesh)
    ref = [oracle_mod.solve_frequency_symmetric(default_oracle_gf, mesh.merged(), st.submesh, st.nb_images,
                                                st.kind in ("reflections", "dihedral"), oracle_mod.rigid_body_dofs(),
                                                w, wave_directions=heads, water_depth=depth) for w in omegas]
    errs = coefficient_errors(res, ref, body.dofs)
    assert max(errs.values()) < 1e-6, errs


def _limit_added_mass_error(res, idx, ref, dofs):
    want = np.array([[ref["added_mass"][i][j] for j in dofs] for i in dofs])
    floor = 1e-3 * np.abs(want).max()
    return float(np.max(np.abs(res.added_mass[idx] - want) / np.maximum(np.abs(want), floor)))


@pytest.mark.parametrize("precision,gate", [("fp64", 1e-7), ("mixed", 1e-5)])
def test_limit_frequencies_in_the_frequency_sweep(oracle_mod, default_oracle_gf, tmp_path, precision, gate):
    """omega = 0 and infinity inside a sweep of B200Engine.solve_frequencies
    (capytaine's pytest/test_bem_zero_and_infinite_freq.py:118-155): added
    mass against the oracle's symbolic-frequency solve, damping exactly zero,
    NaN wave forces, and the finite frequency of the same batch unchanged; in
    finite depth omega = infinity solves and omega = 0 raises."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    from test_gpu_solve import coefficient_errors
    mesh = mesh_sphere(radius=1.0, resolution=(8, 16)).immersed_part()
    body = FloatingBody(mesh, rigid_body_dofs())
    odofs = oracle_mod.rigid_body_dofs()
    eng = B200Engine(green_function=_gpu_gf(default_oracle_gf, tmp_path), precision=precision, max_batch=3)
    res = eng.solve_frequencies(body, [0.0, 1.2, np.inf])
    for idx, omega in ((0, 0.0), (2, np.inf)):
        ref = oracle_mod.solve_radiation_limit_frequency(default_oracle_gf, mesh, odofs, omega)
        assert _limit_added_mass_error(res, idx, ref, list(body.dofs)) < gate, omega
        assert np.all(res.radiation_damping[idx] == 0.0)
        assert np.all(np.isnan(res.excitation[idx]))
    finite = eng.solve_frequencies(body, [1.2])
    same = 1e-9 if precision == "fp64" else 1e-7  # the refinement may take other iteration counts alone
    for name in ("added_mass", "radiation_damping", "excitation"):
        a, b = getattr(res, name)[1], getattr(finite, name)[0]
        assert np.abs(a - b).max() <= same * np.abs(b).max(), name
    res = eng.solve_frequencies(body, [1.0, np.inf], water_depth=5.0)
    ref = oracle_mod.solve_radiation_limit_frequency(default_oracle_gf, mesh, odofs, np.inf, water_depth=5.0)
    assert _limit_added_mass_error(res, 1, ref, list(body.dofs)) < gate
    assert np.all(res.radiation_damping[1] == 0.0)
    first = dataclasses.replace(res, **{k: getattr(res, k)[:1] for k in (
        "omegas", "added_mass", "radiation_damping", "diffraction", "froude_krylov", "excitation")})
    ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh, odofs, 1.0, water_depth=5.0)]
    errs = coefficient_errors(first, ref, body.dofs)
    assert max(errs.values()) < 1e-5, errs
    with pytest.raises(NotImplementedError):
        eng.solve_frequencies(body, [0.0], water_depth=5.0)


def test_limit_frequencies_on_a_symmetric_mesh(oracle_mod, default_oracle_gf, tmp_path):
    """The symmetric sweep at omega = 0 and infinity (the first block column
    assembled by the general kernel at k = 0 and infinity) against the oracle's
    limit solve of the merged mesh, on a mesh whose images are exact."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    from test_symmetry_cpu import _symmetric_cases
    mesh = _symmetric_cases(exact=True)["reflections"]
    body = FloatingBody(mesh, rigid_body_dofs())
    eng = B200Engine(green_function=_gpu_gf(default_oracle_gf, tmp_path), max_batch=2)
    res = eng.solve_frequencies(body, [0.0, np.inf])
    assert res.stats["symmetry"] == "reflections"
    for idx, omega in ((0, 0.0), (1, np.inf)):
        ref = oracle_mod.solve_radiation_limit_frequency(default_oracle_gf, mesh.merged(),
                                                         oracle_mod.rigid_body_dofs(), omega)
        assert _limit_added_mass_error(res, idx, ref, list(body.dofs)) < 1e-6, omega
        assert np.all(res.radiation_damping[idx] == 0.0)
