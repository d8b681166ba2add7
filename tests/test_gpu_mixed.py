"""Mixed-precision solve: float32 tensor-core LU alone (TF32-level accuracy),
float64-residual iterative refinement (1e-10 relative residual), and the
mixed engine's coefficients against the float64 oracle within the 1e-5 gate."""
import ctypes

import numpy as np
import pytest

from capytaine_b200 import _lib
from capytaine_b200.meshes import mesh_sphere, mesh_parallelepiped

pytestmark = pytest.mark.gpu

MIXED_GATE = 1e-5


def _vp(t):
    return ctypes.c_void_p(t.data_ptr() if hasattr(t, "data_ptr") else int(t))


def _bem_matrix_like(n, rng):
    x = rng.uniform(-1, 1, (n, 3))
    d = np.linalg.norm(x[:, None, :] - x[None, :, :], axis=2) + 0.3
    A = (0.2 / n) * (np.exp(1j * d) / d) * rng.uniform(0.5, 1.5, (n, n))
    return A + 0.5 * np.eye(n) + 0.05 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)


def _setup(n, batch, nrhs, seed):
    import torch
    rng = np.random.default_rng(seed)
    lib = _lib.load()
    npad = -(-n // 128) * 128
    mats = [_bem_matrix_like(n, rng) for _ in range(batch)]
    rhs = [rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs)) for _ in range(batch)]
    K = torch.stack([torch.as_tensor(np.ascontiguousarray(m.T)) for m in mats]).cuda()  # column-major n x n
    B = torch.zeros((batch, nrhs, npad), dtype=torch.complex128, device="cuda")
    for b in range(batch):
        B[b, :, :n] = torch.as_tensor(rhs[b].T)
    work = torch.empty(int(lib.bem_clu_workspace_bytes(npad, batch)) + 1024, dtype=torch.uint8, device="cuda")
    wptr = (work.data_ptr() + 1023) // 1024 * 1024
    piv = torch.empty((batch, npad), dtype=torch.int32, device="cuda")
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(lib.bem_clu_factor(_vp(K), n, n * n, n, npad, batch, _vp(piv), _vp(info), _vp(wptr), _vp(err),
                                  _lib.stream_ptr()))
    return lib, npad, mats, rhs, K, B, work, wptr, piv, info, err


@pytest.mark.parametrize("n,batch,nrhs", [(128, 1, 1), (300, 2, 7), (700, 1, 16)])
def test_float32_lu_solve(n, batch, nrhs):
    import torch
    lib, npad, mats, rhs, K, B, work, wptr, piv, info, err = _setup(n, batch, nrhs, n)
    _lib.check(lib.bem_clu_solve(_vp(wptr), npad, batch, _vp(piv), _vp(B), npad, npad * nrhs, nrhs, _vp(err),
                                 _lib.stream_ptr()))
    torch.cuda.synchronize()
    assert info.cpu().tolist() == [0] * batch and int(err.item()) == 0
    for b in range(batch):
        x = B[b, :, :n].T.cpu().numpy()
        ref = np.linalg.solve(mats[b], rhs[b])
        assert np.abs(x - ref).max() / np.abs(ref).max() < 5e-3  # TF32 trailing updates


@pytest.mark.parametrize("n,batch,nrhs", [(300, 2, 7), (1000, 1, 16)])
def test_refinement_reaches_1e10(n, batch, nrhs):
    import torch
    lib, npad, mats, rhs, K, B, work, wptr, piv, info, err = _setup(n, batch, nrhs, n + 1)
    X = torch.zeros_like(B)
    R = torch.zeros_like(B)
    ts = torch.empty(int(lib.bem_zgemm_ts_workspace_bytes(n, n, nrhs, batch)), dtype=torch.uint8, device="cuda")
    norms = torch.zeros(2 * batch * nrhs + 2, dtype=torch.float64, device="cuda")
    iters, resid = ctypes.c_int32(0), ctypes.c_double(0.0)
    _lib.check(lib.bem_refine_solve(_vp(K), n, n * n, n, npad, batch, _vp(wptr), _vp(piv), _vp(B), _vp(X), _vp(R),
                                    npad, npad * nrhs, nrhs, 1e-10, 30, _vp(ts), _vp(norms), _vp(err),
                                    ctypes.byref(iters), ctypes.byref(resid), _lib.stream_ptr()))
    assert resid.value <= 1e-10 and 1 <= iters.value <= 10
    for b in range(batch):  # B is read only
        np.testing.assert_array_equal(B[b, :, :n].T.cpu().numpy(), rhs[b])
    for b in range(batch):
        x = X[b, :, :n].T.cpu().numpy()
        ref = np.linalg.solve(mats[b], rhs[b])
        assert np.abs(x - ref).max() / np.abs(ref).max() < 1e-9


def _shared_table_gf(oracle_gf, tmp_path, **kw):
    import os
    from capytaine_b200.green_function import Delhommeau
    gf = Delhommeau(tabulation_cache_dir=str(tmp_path), **kw)
    np.savez(os.path.join(str(tmp_path), gf._cache_filename), r_range=oracle_gf.tabulated_r_range,
             z_range=oracle_gf.tabulated_z_range, values=oracle_gf.tabulated_integrals)
    return gf


@pytest.mark.parametrize("geometry", ["hemisphere", "barge"])
def test_mixed_engine_against_fp64_oracle(oracle_mod, default_oracle_gf, tmp_path, geometry):
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    from test_gpu_solve import coefficient_errors
    if geometry == "hemisphere":
        mesh = mesh_sphere(radius=1.0, resolution=(12, 24)).immersed_part()
        omegas = np.linspace(0.3, 4.0, 5)
    else:
        mesh = mesh_parallelepiped(size=(16, 4, 4), resolution=(32, 8, 8)).immersed_part()
        omegas = np.linspace(0.2, 2.5, 4)
    body = FloatingBody(mesh, rigid_body_dofs())
    eng = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), precision="mixed", max_batch=3)
    res = eng.solve_frequencies(body, omegas, wave_directions=(0.0, np.pi / 3))
    assert res.stats["refine_residual"] <= 1e-10
    ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh, oracle_mod.rigid_body_dofs(), w,
                                      wave_directions=(0.0, np.pi / 3)) for w in omegas]
    errs = coefficient_errors(res, ref, body.dofs)
    assert max(errs.values()) < MIXED_GATE, errs


def test_float32_wave_term_keeps_added_mass_and_excitation(oracle_mod, default_oracle_gf, tmp_path):
    """The optional float32 wave-term assembly: added mass and excitation stay
    within the gate; radiation damping at low kr does not (documented), so it
    is not the engine default."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    from test_gpu_solve import coefficient_errors
    mesh = mesh_sphere(radius=1.0, resolution=(12, 24)).immersed_part()
    body = FloatingBody(mesh, rigid_body_dofs())
    omegas = np.linspace(0.3, 4.0, 5)
    eng = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), precision="mixed",
                     assembly_precision="mixed")
    res = eng.solve_frequencies(body, omegas)
    ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh, oracle_mod.rigid_body_dofs(), w) for w in omegas]
    errs = coefficient_errors(res, ref, body.dofs)
    assert errs["added_mass"] < MIXED_GATE and errs["excitation"] < MIXED_GATE, errs


def test_refinement_reports_non_convergence():
    """max_iter reached above tol: BEM_ERR_NOT_CONVERGED with the iteration
    count and the residual of the last iterate."""
    import torch
    n, batch, nrhs = 300, 1, 3
    lib, npad, mats, rhs, K, B, work, wptr, piv, info, err = _setup(n, batch, nrhs, 7)
    X, R = torch.zeros_like(B), torch.zeros_like(B)
    ts = torch.empty(int(lib.bem_zgemm_ts_workspace_bytes(n, n, nrhs, batch)), dtype=torch.uint8, device="cuda")
    norms = torch.zeros(2 * batch * nrhs + 2, dtype=torch.float64, device="cuda")
    iters, resid = ctypes.c_int32(0), ctypes.c_double(0.0)
    st = lib.bem_refine_solve(_vp(K), n, n * n, n, npad, batch, _vp(wptr), _vp(piv), _vp(B), _vp(X), _vp(R), npad,
                              npad * nrhs, nrhs, 1e-300, 2, _vp(ts), _vp(norms), _vp(err), ctypes.byref(iters),
                              ctypes.byref(resid), _lib.stream_ptr())
    assert st == _lib.BEM_ERR_NOT_CONVERGED and iters.value == 2 and 0.0 < resid.value < 1e-5
    assert b"iterative refinement stopped" in lib.bem_last_error()


def test_refinement_of_a_column_block_leaves_other_columns_alone():
    """Columns [0, 2) of a 3-column block of 2 matrices (batch stride covers
    all 3): the third column of X and R keeps what it held."""
    import torch
    n, batch, ncol = 300, 2, 3
    lib, npad, mats, rhs, K, B, work, wptr, piv, info, err = _setup(n, batch, ncol, 5)
    X = torch.full_like(B, 3.0)
    R = torch.full_like(B, 5.0)
    ts = torch.empty(int(lib.bem_zgemm_ts_workspace_bytes(n, n, 2, batch)), dtype=torch.uint8, device="cuda")
    norms = torch.zeros(2 * batch * 2 + 2, dtype=torch.float64, device="cuda")
    iters, resid = ctypes.c_int32(0), ctypes.c_double(0.0)
    _lib.check(lib.bem_refine_solve(_vp(K), n, n * n, n, npad, batch, _vp(wptr), _vp(piv), _vp(B), _vp(X), _vp(R),
                                    npad, npad * ncol, 2, 1e-10, 30, _vp(ts), _vp(norms), _vp(err),
                                    ctypes.byref(iters), ctypes.byref(resid), _lib.stream_ptr()))
    assert resid.value <= 1e-10
    assert torch.all(X[:, 2, :] == 3.0) and torch.all(R[:, 2, :] == 5.0)
    for b in range(batch):
        ref = np.linalg.solve(mats[b], rhs[b][:, :2])
        assert np.abs(X[b, :2, :n].T.cpu().numpy() - ref).max() / np.abs(ref).max() < 1e-9
