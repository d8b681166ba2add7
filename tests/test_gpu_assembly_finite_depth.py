"""Finite depth on the device against the CPU oracle: the finite-depth
assembly kernel (bem_assemble_finite_depth, Delhommeau's method of
matrices.f90:197-305 and Green_wave.f90:311-508) and the finite-depth solve
through capytaine's MatrixEngine seam.  Both sides take the same tabulation
(through the cache file) and the same Prony decomposition, so only
floating-point rounding is left in the matrices: 1e-10 relative to the largest
entry, as the infinite-depth float64 path."""
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
