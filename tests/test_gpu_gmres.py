"""Device GMRES against SciPy's, the linear algebra behind capytaine's
solve_gmres (bem/engines.py:74-89), and GMRES-preconditioned refinement of the
float32 LU.

Plain GMRES follows SciPy's iteration step by step (same Arnoldi order, same
rotations, same restart and tolerance rules), so the device iterate matches
SciPy's to rounding and stops after the same number of inner iterations."""
import ctypes

import numpy as np
import pytest

from capytaine_b200 import _lib

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr() if hasattr(t, "data_ptr") else int(t))


def _scipy_gmres(A, b, **kw):
    import scipy.sparse.linalg as ssl
    count = [0]

    def cb(_):
        count[0] += 1
    x, info = ssl.gmres(A, b, callback=cb, callback_type="pr_norm", **kw)
    return x, info, count[0]


def _gmres_device(mats, rhs, *, atol, rtol, restart=20, max_cycles=1000, precond=None, npad=None):
    """mats: batch of (n, n); rhs: batch of (n, nrhs).  Returns X, status, iters, resid."""
    import torch
    lib = _lib.load()
    batch = len(mats)
    n, nrhs = rhs[0].shape
    npad = npad or n
    A = torch.stack([torch.as_tensor(np.ascontiguousarray(m.T)) for m in mats]).cuda()
    B = torch.zeros((batch, nrhs, npad), dtype=torch.complex128, device="cuda")
    for b in range(batch):
        B[b, :, :n] = torch.as_tensor(rhs[b].T)
    X = torch.full_like(B, 7.0)  # overwritten: x0 = 0 inside
    nbytes = int(lib.bem_gmres_workspace_bytes(n, npad, nrhs, batch, restart))
    work = torch.empty(nbytes + 256, dtype=torch.uint8, device="cuda")
    wptr = (work.data_ptr() + 255) // 256 * 256
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    iters, resid = ctypes.c_int32(0), ctypes.c_double(0.0)
    st = lib.bem_gmres_solve(_vp(A), n, n * n, n, npad, batch, _vp(B), _vp(X), npad, npad * nrhs, nrhs, atol, rtol,
                             restart, max_cycles, precond, _vp(wptr), _vp(err), ctypes.byref(iters),
                             ctypes.byref(resid), _lib.stream_ptr())
    torch.cuda.synchronize()
    xs = [X[b, :, :n].T.cpu().numpy() for b in range(batch)]
    return xs, st, iters.value, resid.value, A, B


def _bem_k(n_lat, n_lon, omega):
    """K of the default Delhommeau oracle on a hemisphere: a real BEM system."""
    from oracle import oracle
    from capytaine_b200.meshes import mesh_sphere
    mesh = mesh_sphere(radius=1.0, resolution=(n_lat, n_lon)).immersed_part()
    gf = oracle.OracleDelhommeau(tabulation_nr=328, tabulation_nz=46, tabulation_grid_shape="legacy",
                                 tabulation_nb_integration_points=251)
    _, K = gf.evaluate(mesh, mesh, wavenumber=omega ** 2 / 9.81)
    return mesh, K


def _wave_rhs(mesh, rng, nrhs):
    c = mesh.faces_centers
    cols = [np.exp(1j * (c[:, 0] * np.cos(t) + c[:, 1] * np.sin(t))) * np.exp(c[:, 2]) * mesh.faces_normals[:, 2]
            for t in rng.uniform(0, 2 * np.pi, nrhs)]
    return np.stack(cols, axis=1)


def test_plain_gmres_follows_scipy_on_a_bem_matrix():
    rng = np.random.default_rng(3)
    mesh, K = _bem_k(10, 20, 1.5)
    b = _wave_rhs(mesh, rng, 3)
    xs, st, iters, resid, *_ = _gmres_device([K], [b], atol=1e-6, rtol=1e-5)
    assert st == _lib.BEM_OK
    ref_iters = []
    for c in range(b.shape[1]):
        xr, info, nit = _scipy_gmres(K, b[:, c], atol=1e-6)
        assert info == 0
        ref_iters.append(nit)
        assert np.abs(xs[0][:, c] - xr).max() <= 1e-9 * np.abs(xr).max()
        assert np.linalg.norm(b[:, c] - K @ xs[0][:, c]) <= max(1e-6, 1e-5 * np.linalg.norm(b[:, c]))
    assert iters == max(ref_iters)


def test_plain_gmres_batched_with_restarts():
    """Several matrices and columns in one call, restart 5 so that the inner
    tolerance adaptation and several cycles are exercised."""
    rng = np.random.default_rng(5)
    mats, rhs = [], []
    for w in (0.8, 2.2):
        mesh, K = _bem_k(8, 16, w)
        mats.append(K)
        rhs.append(_wave_rhs(mesh, rng, 4))
    xs, st, iters, resid, *_ = _gmres_device(mats, rhs, atol=0.0, rtol=1e-9, restart=5)
    assert st == _lib.BEM_OK and resid <= 1e-9
    for K, b, x in zip(mats, rhs, xs):
        for c in range(b.shape[1]):
            xr, info, _ = _scipy_gmres(K, b[:, c], atol=0.0, rtol=1e-9, restart=5)
            assert info == 0
            assert np.abs(x[:, c] - xr).max() <= 1e-7 * np.abs(xr).max()
            xe = np.linalg.solve(K, b[:, c])
            assert np.abs(x[:, c] - xe).max() <= 1e-7 * np.abs(xe).max()


def test_zero_rhs_and_non_convergence():
    import torch
    rng = np.random.default_rng(11)
    mesh, K = _bem_k(8, 16, 1.0)
    b = _wave_rhs(mesh, rng, 2)
    b[:, 1] = 0.0
    xs, st, iters, resid, *_ = _gmres_device([K], [b], atol=0.0, rtol=1e-5)
    assert st == _lib.BEM_OK and np.all(xs[0][:, 1] == 0)
    # one cycle of two iterations cannot reach 1e-14
    xs, st, iters, resid, *_ = _gmres_device([K], [b[:, :1]], atol=0.0, rtol=1e-14, restart=2, max_cycles=1)
    assert st == _lib.BEM_ERR_NOT_CONVERGED and iters == 2 and resid > 1e-14
    assert b"No convergence of the GMRES" in _lib.load().bem_last_error()


@pytest.mark.parametrize("n,batch,nrhs", [(300, 2, 7), (1000, 1, 16)])
def test_gmres_preconditioned_by_float32_lu_reaches_1e10(n, batch, nrhs):
    from test_gpu_mixed import _setup
    lib, npad, mats, rhs, K, B, work, wptr, piv, info, err = _setup(n, batch, nrhs, n + 3)
    xs, st, iters, resid, *_ = _gmres_device(mats, rhs, atol=0.0, rtol=1e-10, precond=_vp(wptr), npad=npad)
    assert st == _lib.BEM_OK and resid <= 1e-10 and 1 <= iters <= 8
    for b in range(batch):
        ref = np.linalg.solve(mats[b], rhs[b])
        assert np.abs(xs[b] - ref).max() / np.abs(ref).max() < 1e-9


def test_engines_with_gmres_against_oracle(oracle_mod, default_oracle_gf, tmp_path):
    """linear_solver='gmres' (float64) against the oracle solved with SciPy's
    GMRES, and the mixed engine with GMRES refinement against the LU oracle."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.meshes import mesh_sphere
    from test_gpu_mixed import _shared_table_gf
    from test_gpu_solve import coefficient_errors
    mesh = mesh_sphere(radius=1.0, resolution=(10, 20)).immersed_part()
    body = FloatingBody(mesh, rigid_body_dofs())
    omegas = np.array([0.5, 1.7, 3.0])
    gf = _shared_table_gf(default_oracle_gf, tmp_path)
    ref_gmres = [oracle_mod.solve_frequency(default_oracle_gf, mesh, oracle_mod.rigid_body_dofs(), w,
                                            linear_solver="gmres") for w in omegas]
    ref_lu = [oracle_mod.solve_frequency(default_oracle_gf, mesh, oracle_mod.rigid_body_dofs(), w) for w in omegas]
    res = B200Engine(green_function=gf, linear_solver="gmres").solve_frequencies(body, omegas)
    assert res.stats["gmres_iters"] >= 1
    errs = coefficient_errors(res, ref_gmres, body.dofs)
    assert max(errs.values()) < 1e-6, errs  # same iteration, same stopping point as SciPy
    res = B200Engine(green_function=gf, precision="mixed", refinement="gmres").solve_frequencies(body, omegas)
    assert res.stats["refine_residual"] <= 1e-10
    errs = coefficient_errors(res, ref_lu, body.dofs)
    assert max(errs.values()) < 1e-7, errs


def test_refinement_stops_and_gmres_recovers_near_a_singular_matrix():
    """K with one eigenvalue 1e-7 (what an irregular frequency does to the BEM
    system): the float32 LU is wrong in that direction, the classical iteration
    x += (LU)^-1 r no longer contracts and stops early as non-converged; GMRES
    right-preconditioned by the same factors removes the outlier in a few
    iterations.  The factors are then close to singular themselves (|M^-1| of
    order 1e5-1e6), where the float32 substitutions are measurably nonlinear:
    the flexible form (M^-1 v_k kept for the update of x) converges in about 6
    iterations, the plain form (M^-1 applied again to V y) took over 80.  The
    tolerance is 1e-8: with |x| ~ 1e7 |b| the float64 residual b - K x cannot
    be resolved much below ~1e-10 |b|."""
    import torch
    rng = np.random.default_rng(21)
    n, nrhs = 256, 3
    npad = 256
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    lam = rng.uniform(0.5, 1.5, n) * np.exp(1j * rng.uniform(-0.3, 0.3, n))
    lam[0] = 1e-7 * (1 + 1j)
    A = (Q * lam) @ Q.conj().T
    b = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    lib = _lib.load()
    K = torch.as_tensor(np.ascontiguousarray(A.T)).cuda().reshape(1, -1)
    work = torch.empty(int(lib.bem_clu_workspace_bytes(npad, 1)) + 1024, dtype=torch.uint8, device="cuda")
    wptr = (work.data_ptr() + 1023) // 1024 * 1024
    piv = torch.empty((1, npad), dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(lib.bem_clu_factor(_vp(K), n, n * n, n, npad, 1, _vp(piv), _vp(info), _vp(wptr), _vp(err),
                                  _lib.stream_ptr()))
    B = torch.zeros((1, nrhs, npad), dtype=torch.complex128, device="cuda")
    B[0, :, :n] = torch.as_tensor(b.T)
    X, R = torch.zeros_like(B), torch.zeros_like(B)
    ts = torch.empty(int(lib.bem_zgemm_ts_workspace_bytes(n, n, nrhs, 1)), dtype=torch.uint8, device="cuda")
    norms = torch.zeros(2 * nrhs + 2, dtype=torch.float64, device="cuda")
    iters, resid = ctypes.c_int32(0), ctypes.c_double(0.0)
    st = lib.bem_refine_solve(_vp(K), n, n * n, n, npad, 1, _vp(wptr), _vp(piv), _vp(B), _vp(X), _vp(R), npad,
                              npad * nrhs, nrhs, 1e-8, 30, _vp(ts), _vp(norms), _vp(err), ctypes.byref(iters),
                              ctypes.byref(resid), _lib.stream_ptr())
    assert st == _lib.BEM_ERR_NOT_CONVERGED and iters.value < 30, (st, iters.value, resid.value)
    xs, st, it, res, *_ = _gmres_device([A], [b], atol=0.0, rtol=1e-8, precond=_vp(wptr), npad=npad)
    assert st == _lib.BEM_OK and res <= 1e-8 and it <= 20, (st, it, res, _lib.load().bem_last_error())
    for c in range(nrhs):
        assert np.linalg.norm(b[:, c] - A @ xs[0][:, c]) <= 2e-8 * np.linalg.norm(b[:, c])


def test_flexible_gmres_over_short_restart_cycles():
    """The preconditioned vectors are kept per restart cycle: with restart 2 a
    K with one eigenvalue 1e-6 and a regular K, factored together by the
    float32 LU and solved in one batched call, converge over several cycles,
    every column to 1e-9 of its right-hand side (|x| reaches 1e6 |b| for the
    first, so the float64 residual still resolves 1e-9)."""
    import torch
    rng = np.random.default_rng(8)
    n, nrhs, npad = 256, 4, 256
    mats = []
    for lam0 in (1e-6 * (1 - 1j), None):
        Q, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
        lam = rng.uniform(0.5, 1.5, n) * np.exp(1j * rng.uniform(-0.3, 0.3, n))
        if lam0 is not None:
            lam[0] = lam0
        mats.append((Q * lam) @ Q.conj().T)
    rhs = [rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs)) for _ in mats]
    lib = _lib.load()
    K = torch.stack([torch.as_tensor(np.ascontiguousarray(A.T)).reshape(-1) for A in mats]).cuda()
    work = torch.empty(int(lib.bem_clu_workspace_bytes(npad, 2)) + 1024, dtype=torch.uint8, device="cuda")
    wptr = (work.data_ptr() + 1023) // 1024 * 1024
    piv = torch.empty((2, npad), dtype=torch.int32, device="cuda")
    info = torch.zeros(2, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(lib.bem_clu_factor(_vp(K), n, n * n, n, npad, 2, _vp(piv), _vp(info), _vp(wptr), _vp(err),
                                  _lib.stream_ptr()))
    xs, st, it, res, *_ = _gmres_device(mats, rhs, atol=0.0, rtol=1e-9, restart=2, precond=_vp(wptr), npad=npad)
    assert st == _lib.BEM_OK and res <= 1e-9, (st, it, res, _lib.load().bem_last_error())
    assert it > 2  # more than one cycle of 2
    for A, b, x in zip(mats, rhs, xs):
        for c in range(nrhs):
            assert np.linalg.norm(b[:, c] - A @ x[:, c]) <= 2e-9 * np.linalg.norm(b[:, c])
