"""Dense linear algebra and frequency solves on the GPU against NumPy/SciPy
(the reference's own linear algebra) and against the CPU oracle."""
import ctypes

import numpy as np
import pytest

from capytaine_b200 import _lib
from capytaine_b200.meshes import mesh_sphere

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _bem_matrix_like(n, rng):
    """Complex matrix with the structure of K: 1/2 on the diagonal plus a
    smooth dense part (well conditioned, no dominant pivot pattern)."""
    x = rng.uniform(-1, 1, (n, 3))
    d = np.linalg.norm(x[:, None, :] - x[None, :, :], axis=2) + 0.3
    A = (0.2 / n) * (np.exp(1j * d) / d) * rng.uniform(0.5, 1.5, (n, n))
    return A + 0.5 * np.eye(n) + 0.05 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)


@pytest.mark.parametrize("n,batch,nrhs", [(64, 1, 1), (200, 3, 7), (300, 2, 64)])
def test_lu_solve_matches_numpy(n, batch, nrhs):
    import torch
    rng = np.random.default_rng(n)
    lib = _lib.load()
    npad = -(-n // 64) * 64
    mats = [_bem_matrix_like(n, rng) for _ in range(batch)]
    rhs = [rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs)) for _ in range(batch)]
    A = torch.zeros((batch, npad, npad), dtype=torch.complex128, device="cuda")
    Bt = torch.zeros((batch, nrhs, npad), dtype=torch.complex128, device="cuda")
    for b in range(batch):
        A[b].T[:n, :n] = torch.as_tensor(mats[b])
        Bt[b, :, :n] = torch.as_tensor(rhs[b].T)
    s = _lib.stream_ptr()
    _lib.check(lib.bem_zpad_identity(_vp(A), npad, npad * npad, batch, n, npad, s))
    piv = torch.empty((batch, npad), dtype=torch.int32, device="cuda")
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    work = torch.empty(int(lib.bem_zlu_workspace_bytes(npad, batch)), dtype=torch.uint8, device="cuda")
    _lib.check(lib.bem_zlu_factor(_vp(A), npad, npad, npad * npad, batch, _vp(piv), _vp(info), _vp(work), s))
    _lib.check(lib.bem_zlu_solve(_vp(A), npad, npad, npad * npad, batch, _vp(piv), _vp(work), _vp(Bt), npad,
                                 npad * nrhs, nrhs, _vp(err), s))
    torch.cuda.synchronize()
    assert info.cpu().numpy().tolist() == [0] * batch
    assert int(err.item()) == 0
    for b in range(batch):
        x = Bt[b, :, :n].T.cpu().numpy()
        ref = np.linalg.solve(mats[b], rhs[b])
        assert np.abs(x - ref).max() / np.abs(ref).max() < 1e-12
        # padded rows stay zero
        if npad > n:
            assert np.abs(Bt[b, :, n:].cpu().numpy()).max() == 0.0


def test_zero_pivot_reported():
    import torch
    lib = _lib.load()
    n = 64
    A = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
    A.T[:, :] = torch.eye(n, dtype=torch.complex128)
    A.T[5, :] = 0  # singular: a zero row
    piv = torch.empty(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    work = torch.empty(int(lib.bem_zlu_workspace_bytes(n, 1)), dtype=torch.uint8, device="cuda")
    _lib.check(lib.bem_zlu_factor(_vp(A), n, n, n * n, 1, _vp(piv), _vp(info), _vp(work), _lib.stream_ptr()))
    assert int(info.item()) == 6


@pytest.mark.parametrize("M,N,K", [(64, 64, 64), (130, 70, 33), (257, 256, 64)])
def test_zgemm_matches_numpy(M, N, K):
    import torch
    rng = np.random.default_rng(M + N + K)
    lib = _lib.load()
    a = rng.standard_normal((M, K)) + 1j * rng.standard_normal((M, K))
    b = rng.standard_normal((K, N)) + 1j * rng.standard_normal((K, N))
    c = rng.standard_normal((M, N)) + 1j * rng.standard_normal((M, N))
    At = torch.as_tensor(a.T.copy(), device="cuda")   # column-major M x K
    Bt = torch.as_tensor(b.T.copy(), device="cuda")
    Ct = torch.as_tensor(c.T.copy(), device="cuda")
    _lib.check(lib.bem_zgemm(M, N, K, -1.0, _vp(At), M, 0, _vp(Bt), K, 0, 1.0, _vp(Ct), M, 0, 1, _lib.stream_ptr()))
    ref = c - a @ b
    got = Ct.T.cpu().numpy()
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-13


@pytest.mark.parametrize("M,K,nrhs", [(100, 100, 1), (700, 650, 7), (1000, 3000, 16)])
def test_zgemm_ts_matches_numpy(M, K, nrhs):
    import torch
    rng = np.random.default_rng(M)
    lib = _lib.load()
    a = rng.standard_normal((M, K)) + 1j * rng.standard_normal((M, K))
    x = rng.standard_normal((K, nrhs)) + 1j * rng.standard_normal((K, nrhs))
    y = rng.standard_normal((M, nrhs)) + 1j * rng.standard_normal((M, nrhs))
    At = torch.as_tensor(a.T.copy(), device="cuda")
    Xt = torch.as_tensor(x.T.copy(), device="cuda")
    Yt = torch.as_tensor(y.T.copy(), device="cuda")
    work = torch.empty(int(lib.bem_zgemm_ts_workspace_bytes(M, K, nrhs, 1)), dtype=torch.uint8, device="cuda")
    _lib.check(lib.bem_zgemm_ts(M, K, nrhs, 0.5, -2.0, _vp(At), M, 0, _vp(Xt), K, 0, 1.0, 1.0, _vp(Yt), M, 0, 1,
                                _vp(work), _lib.stream_ptr()))
    ref = (0.5 - 2j) * (a @ x) + (1 + 1j) * y
    assert np.abs(Yt.T.cpu().numpy() - ref).max() / np.abs(ref).max() < 1e-13


def _shared_table_gf(oracle_gf, tmp_path, **kw):
    import os
    from capytaine_b200.green_function import Delhommeau
    gf = Delhommeau(tabulation_cache_dir=str(tmp_path), **kw)
    np.savez(os.path.join(str(tmp_path), gf._cache_filename), r_range=oracle_gf.tabulated_r_range,
             z_range=oracle_gf.tabulated_z_range, values=oracle_gf.tabulated_integrals)
    return gf


def coefficient_errors(res, ref_list, body_dofs):
    """Max relative error per coefficient family, with the floor of
    1e-3 * max |coefficient| against entries that vanish by symmetry."""
    dofs = list(body_dofs)
    A = np.array([[[r["added_mass"][i][j] for j in dofs] for i in dofs] for r in ref_list])
    Bd = np.array([[[r["radiation_damping"][i][j] for j in dofs] for i in dofs] for r in ref_list])
    E = np.array([[[r["excitation"][h][j] for j in dofs] for h in r["excitation"]] for r in ref_list])
    out = {}
    for name, got, ref in (("added_mass", res.added_mass, A), ("radiation_damping", res.radiation_damping, Bd),
                           ("excitation", res.excitation, E)):
        floor = 1e-3 * np.abs(ref).max(axis=tuple(range(1, ref.ndim)), keepdims=True)
        out[name] = float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), floor)))
    return out


def test_frequency_solve_matches_oracle_hemisphere(oracle_mod, default_oracle_gf, tmp_path):
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    mesh = mesh_sphere(radius=1.0, resolution=(12, 24)).immersed_part()
    body = FloatingBody(mesh, rigid_body_dofs())
    omegas = np.linspace(0.3, 4.0, 5)
    eng = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), max_batch=3)
    res = eng.solve_frequencies(body, omegas, wave_directions=(0.0, np.pi / 3))
    odofs = oracle_mod.rigid_body_dofs()
    ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh, odofs, w, wave_directions=(0.0, np.pi / 3))
           for w in omegas]
    errs = coefficient_errors(res, ref, body.dofs)
    assert max(errs.values()) < 1e-9, errs


def test_nemoh2_golden_through_gpu_engine(legacy_oracle_gf, golden, tmp_path):
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    from conftest import hemisphere_volume
    gf = _shared_table_gf(legacy_oracle_gf, tmp_path, tabulation_nr=328, tabulation_nz=46,
                          tabulation_grid_shape="legacy", tabulation_nb_integration_points=251,
                          gf_singularities="high_freq")
    sphere = mesh_sphere(radius=1.0, resolution=(6, 12)).immersed_part()
    body = FloatingBody(sphere, rigid_body_dofs(only=["Heave"]))
    res = B200Engine(green_function=gf).solve_frequencies(body, [1.0, 2.0])
    atol = 1e-3 * hemisphere_volume(sphere) * 1000.0
    for i, key in enumerate(["omega_1", "omega_2"]):
        ref = golden["floating_sphere"][key]
        assert np.isclose(res.added_mass[i, 0, 0], ref["added_mass"], atol=atol)
        assert np.isclose(res.radiation_damping[i, 0, 0], ref["damping"], atol=atol)
        mod, phase = ref["diffraction_force_polar"]
        assert np.isclose(res.diffraction[i, 0, 0], mod * np.exp(1j * phase), rtol=1e-3)


def test_gpu_built_table_end_to_end(oracle_mod, default_oracle_gf):
    """Config-1 shape on a coarser hemisphere: GPU-built table, every stage on
    the GPU, coefficients within the 1e-6 gate of the float64 path."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.green_function import Delhommeau
    mesh = mesh_sphere(radius=1.0, resolution=(20, 40)).immersed_part()
    body = FloatingBody(mesh, rigid_body_dofs(only=["Heave"]))
    omegas = np.linspace(0.1, 5.0, 6)
    res = B200Engine(green_function=Delhommeau(tabulation_cache_dir=None)).solve_frequencies(body, omegas)
    ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh, oracle_mod.rigid_body_dofs(only=["Heave"]), w)
           for w in omegas]
    errs = coefficient_errors(res, ref, body.dofs)
    assert max(errs.values()) < 1e-6, errs


def test_matrix_engine_interface(default_oracle_gf, tmp_path):
    """build_matrices / linear_solver / S @ x as capytaine's BEMSolver calls them
    (bem/solver.py:188-199)."""
    from capytaine_b200.engine import B200Engine
    mesh = mesh_sphere(resolution=(8, 12)).immersed_part()
    eng = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path))
    S, K = eng.build_matrices(mesh, mesh, free_surface=0.0, water_depth=np.inf, wavenumber=1.0,
                              adjoint_double_layer=True, diagonal_term_in_double_layer=True)
    assert eng.build_matrices(mesh, mesh, free_surface=0.0, water_depth=np.inf, wavenumber=1.0,
                              adjoint_double_layer=True, diagonal_term_in_double_layer=True)[1] is K
    assert K.dtype == np.complex128 and K.shape == (mesh.nb_faces, mesh.nb_faces)
    rng = np.random.default_rng(1)
    b = rng.standard_normal(mesh.nb_faces) + 1j * rng.standard_normal(mesh.nb_faces)
    x = eng.linear_solver(K, b)
    Kh, Sh = np.asarray(K), np.asarray(S)
    assert np.abs(Kh @ x - b).max() < 1e-10 * np.abs(b).max()
    assert np.allclose(S @ x, Sh @ x, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_direct_method_against_oracle(oracle_mod, default_oracle_gf, tmp_path, precision):
    """method='direct' (potential = D^-1 S bc, bem/solver.py:172-187) against the
    oracle's direct solve, and close to the indirect method as the reference's
    test_bem_solver.py:77-83 asks (same forces within 10%)."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    mesh = mesh_sphere(radius=1.0, resolution=(12, 24)).immersed_part()
    body = FloatingBody(mesh, rigid_body_dofs())
    omegas = np.array([0.6, 1.0, 2.2])
    gf = _shared_table_gf(default_oracle_gf, tmp_path)
    direct = B200Engine(green_function=gf, precision=precision, method="direct").solve_frequencies(body, omegas)
    ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh, oracle_mod.rigid_body_dofs(), w, method="direct")
           for w in omegas]
    errs = coefficient_errors(direct, ref, body.dofs)
    assert max(errs.values()) < (1e-6 if precision == "fp64" else 1e-5), errs
    indirect = B200Engine(green_function=gf, precision=precision).solve_frequencies(body, omegas)
    surge = list(body.dofs).index("Surge")
    np.testing.assert_allclose(np.abs(direct.excitation[:, 0, surge]), np.abs(indirect.excitation[:, 0, surge]),
                               rtol=1e-1)
