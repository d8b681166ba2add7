"""Finite depth and limit frequencies on the device against the CPU oracle.

* The finite-depth assembly kernel (bem_assemble_finite_depth, Delhommeau's
  method of matrices.f90:197-305 and Green_wave.f90:311-508): both sides take
  the same tabulation (through the cache file) and the same Prony
  decomposition, so only floating-point rounding is left: 1e-10 relative to
  the largest entry, as the infinite-depth float64 path (1e-6 for complex64
  outputs).
* Finite-depth solves: through capytaine's MatrixEngine seam, and through
  B200Engine.solve_frequencies (dense and symmetric meshes, float64 and mixed
  engines) with the finite-depth Airy right-hand sides, at the gates of the
  frequency-solve metric.
* omega = 0 and infinity inside frequency sweeps, against the oracle's
  symbolic-frequency radiation solve."""
import dataclasses
import os

import numpy as np
import pytest

from capytaine_b200.meshes import Mesh, mesh_rectangle, mesh_sphere

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-10


def _gpu_gf(oracle_gf, tmp_path, **kwargs):
    from capytaine_b200.green_function import Delhommeau
    gf = Delhommeau(tabulation_cache_dir=str(tmp_path), **kwargs)
    np.savez(os.path.join(str(tmp_path), gf._cache_filename), r_range=oracle_gf.tabulated_r_range,
             z_range=oracle_gf.tabulated_z_range, values=oracle_gf.tabulated_integrals)
    return gf


def _close(a, b, rtol):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max() / scale
    assert err <= rtol, f"max error {err:.3e} relative to max |entry| {scale:.3e}"


def _hemisphere(res=(6, 8)):
    return mesh_sphere(resolution=res).immersed_part()


CASES = {
    # (mesh, depth, k, method, gf_singularities, evaluate keywords)
    "newer_lowfreq": (lambda: _hemisphere(), 5.0, 1.0, "newer", "low_freq", {}),
    "newer_highfreq": (lambda: _hemisphere(), 3.0, 0.8, "newer", "high_freq", {}),
    "legacy": (lambda: _hemisphere(), 4.0, 0.5, "legacy", "low_freq", {}),
    "legacy_forces_low_freq": (lambda: _hemisphere(), 4.0, 0.5, "legacy", "high_freq", {}),
    "direct_D": (lambda: _hemisphere(), 5.0, 1.2, "newer", "low_freq", dict(adjoint_double_layer=False)),
    "shallow": (lambda: _hemisphere(), 1.5, 0.3, "newer", "low_freq", {}),
    "deep_water_large_kh": (lambda: _hemisphere(), 20.0, 2.0, "newer", "low_freq", {}),
    "no_diagonal_term": (lambda: _hemisphere(), 5.0, 1.0, "newer", "low_freq",
                         dict(diagonal_term_in_double_layer=False)),
    "full_gradient": (lambda: _hemisphere(), 5.0, 1.0, "newer", "low_freq", dict(early_dot_product=False)),
    "direct_full_gradient": (lambda: _hemisphere(), 3.0, 0.7, "newer", "high_freq",
                             dict(early_dot_product=False, adjoint_double_layer=False)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_finite_depth_assembly_matches_oracle(oracle_mod, default_oracle_gf, tmp_path, name):
    make_mesh, depth, k, method, sing, kw = CASES[name]
    mesh = make_mesh()
    ora = oracle_mod.OracleDelhommeau(gf_singularities=sing, tabulation=default_oracle_gf.tabulation,
                                      finite_depth_method=method)
    gf = _gpu_gf(default_oracle_gf, tmp_path, gf_singularities=sing, finite_depth_method=method)
    decomposition = gf.find_best_exponential_decomposition(k * depth)
    S_ref, K_ref = ora.evaluate(mesh, mesh, wavenumber=k, water_depth=depth, prony=decomposition, **kw)
    S, K = gf.evaluate(mesh, mesh, wavenumber=k, water_depth=depth, **kw)
    assert S.dtype == np.complex128 and K.dtype == np.complex128
    _close(S, S_ref, FP64_RTOL)
    _close(K, K_ref, FP64_RTOL)


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


def test_finite_depth_free_surface_panels_and_points(oracle_mod, default_oracle_gf, tmp_path):
    """Panels on the free surface (a lid) and raw points, some near the sea
    bottom, against the mesh."""
    lid = mesh_rectangle(size=(0.8, 0.8), resolution=(2, 2), center=(0, 0, 0), normal=(0, 0, 1))
    mesh = Mesh.join_meshes(_hemisphere(), lid)
    depth, k = 3.0, 1.5
    gf = _gpu_gf(default_oracle_gf, tmp_path)
    decomposition = gf.find_best_exponential_decomposition(k * depth)
    S_ref, K_ref = default_oracle_gf.evaluate(mesh, mesh, wavenumber=k, water_depth=depth, prony=decomposition)
    S, K = gf.evaluate(mesh, mesh, wavenumber=k, water_depth=depth)
    _close(S, S_ref, FP64_RTOL)
    _close(K, K_ref, FP64_RTOL)
    rng = np.random.default_rng(3)
    pts = np.concatenate([rng.uniform(-2, 2, (30, 3)) * [1, 1, 0] + [0, 0, -0.4],
                          [[0.2, 0.1, -2.95], [4.0, -3.0, -2.5], [30.0, 0.0, -1.0]]])
    S_ref, K_ref = default_oracle_gf.evaluate(pts, mesh, wavenumber=k, water_depth=depth, prony=decomposition)
    S, K = gf.evaluate(pts, mesh, wavenumber=k, water_depth=depth)
    _close(S, S_ref, FP64_RTOL)
    _close(K, K_ref, FP64_RTOL)


def test_finite_depth_sweep_writes_every_wavenumber(oracle_mod, default_oracle_gf, tmp_path):
    """assemble_into with a sweep: one decomposition and one launch per
    wavenumber, each into its own slot."""
    import torch
    mesh = _hemisphere((4, 6))
    depth, ks = 6.0, [0.4, 1.1]
    n = mesh.nb_faces
    gf = _gpu_gf(default_oracle_gf, tmp_path)
    S = torch.zeros((len(ks), n, n), dtype=torch.complex128, device="cuda")
    K = torch.zeros_like(S)
    gf.assemble_into(mesh, mesh, S[0], K[0], water_depth=depth, wavenumber=ks[0], sweep=(ks, n * n, n * n))
    torch.cuda.synchronize()
    for i, k in enumerate(ks):
        S_ref, K_ref = default_oracle_gf.evaluate(mesh, mesh, wavenumber=k, water_depth=depth,
                                                  prony=gf.find_best_exponential_decomposition(k * depth))
        _close(S[i].T.cpu().numpy(), S_ref, FP64_RTOL)
        _close(K[i].T.cpu().numpy(), K_ref, FP64_RTOL)


def _matrix_engine(oracle_gf, tmp_path):
    from capytaine_b200.engine import B200Engine
    return B200Engine(green_function=_gpu_gf(oracle_gf, tmp_path))


def _coefficient_error(value, ref, scale):
    return abs(value - ref) / max(abs(ref), 1e-3 * scale)


@pytest.mark.parametrize("depth,omega", [(4.0, 1.3), (1.5, 0.8)])
def test_finite_depth_solve_through_matrix_engine(oracle_mod, default_oracle_gf, tmp_path, depth, omega):
    """capytaine's BEMSolver in finite depth over this engine (bem/solver.py:188-207):
    build_matrices(water_depth=h) through the finite-depth kernel, then
    linear_solver and S @ sigma on the device, with the radiation and
    finite-depth diffraction right-hand sides the reference's problems build
    (problems_and_results.py:373-381,440-449, airy_waves.py:56-95); added mass,
    damping and excitation against the oracle's finite-depth solve."""
    mesh = mesh_sphere(resolution=(8, 12)).immersed_part()
    dofs = oracle_mod.rigid_body_dofs(only=["Surge", "Heave", "Pitch"])
    rho, g = 1000.0, 9.81
    eng = _matrix_engine(default_oracle_gf, tmp_path)
    k = oracle_mod.finite_depth_wavenumber(omega, depth, g)
    S, K = eng.build_matrices(mesh, mesh, free_surface=0.0, water_depth=depth, wavenumber=k,
                              adjoint_double_layer=True, diagonal_term_in_double_layer=True)
    ref = oracle_mod.solve_frequency(default_oracle_gf, mesh, dofs, omega, water_depth=depth)
    centers, normals = mesh.faces_centers, mesh.faces_normals

    def forces(bc):
        sigma = eng.linear_solver(K, bc)
        return oracle_mod.integrate_pressure(mesh, dofs, 1j * omega * rho * (S @ sigma))

    added, damping = {}, {}
    for name, dof in dofs.items():
        f = forces(-1j * omega * np.sum(dof.motion(centers) * normals, axis=1))
        added[name] = {d: np.real(v) / omega ** 2 for d, v in f.items()}
        damping[name] = {d: np.imag(v) / omega for d, v in f.items()}
    diffraction = forces(-(oracle_mod.airy_waves_velocity(centers, omega, k, g, 0.0, depth) * normals).sum(axis=1))
    for got, want in ((added, ref["added_mass"]), (damping, ref["radiation_damping"])):
        scale = max(abs(v) for row in want.values() for v in row.values())
        errs = [_coefficient_error(got[r][c], want[r][c], scale) for r in want for c in want[r]]
        assert max(errs) < 1e-7, errs
    want = ref["diffraction"][0.0]
    scale = max(abs(v) for v in want.values())
    errs = [_coefficient_error(diffraction[d], want[d], scale) for d in want]
    assert max(errs) < 1e-7, errs


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
