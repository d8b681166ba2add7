"""Safety of the device solves.

* The float64 LU pivots inside its 64-row diagonal blocks only, where LAPACK's
  zgetrf (behind scipy.linalg.lu_factor, capytaine
  tools/block_circulant_matrices.py:374-385) searches the whole column.  Every
  float64 solve therefore checks its residual against the unfactored matrix
  and refines it (bem_zlu_refine_solve).  Matrices whose correct pivots lie
  outside the diagonal blocks (rows of a diagonally dominant matrix moved to
  other blocks) must still match numpy's solve to 1e-12 (normwise, per right-hand side), or
  be flagged.
* The flag waits of the persistent block substitutions are bounded: with one
  block row's completion flag withheld, the waits on it run out, the kernel
  reports BEM_ERR_TIMEOUT through the error flag, and the stream stays usable.
"""
import ctypes

import numpy as np
import pytest

from capytaine_b200 import _lib

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr() if hasattr(t, "data_ptr") else int(t))


def _dominant(n, rng):
    return 10.0 * np.eye(n) + 0.05 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))


PERMUTATIONS = {
    # row i of K is row (i + 32) mod n of the dominant matrix: every diagonal
    # block of K holds half of its large entries in the block to its right
    "cyclic_shift_32": lambda n: (np.arange(n) + 32) % n,
    # rows in reverse order: the large entries sit on the anti-diagonal
    "reversed": lambda n: np.arange(n)[::-1].copy(),
    # each pair of consecutive 64-row blocks swapped
    "block_swap": lambda n: np.arange(n).reshape(-1, 2, 64)[:, ::-1, :].reshape(-1),
}


@pytest.mark.parametrize("perm", sorted(PERMUTATIONS))
@pytest.mark.parametrize("n", [256, 640])
def test_fp64_solve_with_off_block_pivots(perm, n):
    from capytaine_b200.engine import B200Engine, DeviceMatrix, _to_device
    rng = np.random.default_rng(n + len(perm))
    K = _dominant(n, rng)[PERMUTATIONS[perm](n)]
    b = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
    ref = np.linalg.solve(K, b)
    eng = B200Engine(precision="fp64")
    try:
        x = eng.linear_solver(DeviceMatrix(_to_device(np.asfortranarray(K), eng.device), eng), b)
    except (_lib.NotConvergedError, _lib.SingularMatrixError):
        return  # flagged: acceptable, never a silent loss
    # normwise relative error per right-hand side (the residual test is normwise)
    assert np.max(np.linalg.norm(x - ref, axis=0) / np.linalg.norm(ref, axis=0)) < 1e-12, perm


def test_fp64_refined_solve_through_the_c_abi():
    """bem_zlu_refine_solve on a batch: one well-pivoted matrix (one
    iteration) and one whose pivots lie outside the diagonal blocks."""
    import torch
    lib = _lib.load()
    rng = np.random.default_rng(5)
    n, npad, nrhs, batch = 300, 320, 5, 2
    mats = [_dominant(n, rng), _dominant(n, rng)[(np.arange(n) + 32) % n]]
    rhs = [rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs)) for _ in range(batch)]
    K = torch.zeros((batch, n, n), dtype=torch.complex128, device="cuda")  # K[b].T column-major n x n
    LU = torch.zeros((batch, npad, npad), dtype=torch.complex128, device="cuda")
    B = torch.zeros((batch, nrhs, npad), dtype=torch.complex128, device="cuda")
    for i in range(batch):
        K[i].T[:, :] = torch.as_tensor(mats[i])
        LU[i].T[:n, :n] = torch.as_tensor(mats[i])
        B[i, :, :n] = torch.as_tensor(rhs[i].T)
    X, R = torch.zeros_like(B), torch.zeros_like(B)
    s = _lib.stream_ptr()
    piv = torch.empty((batch, npad), dtype=torch.int32, device="cuda")
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    work = torch.empty(int(lib.bem_zlu_workspace_bytes(npad, batch)), dtype=torch.uint8, device="cuda")
    ts = torch.empty(int(lib.bem_zgemm_ts_workspace_bytes(n, n, nrhs, batch)), dtype=torch.uint8, device="cuda")
    norms = torch.zeros(2 * batch * nrhs + 2, dtype=torch.float64, device="cuda")
    _lib.check(lib.bem_zpad_identity(_vp(LU), npad, npad * npad, batch, n, npad, s))
    _lib.check(lib.bem_zlu_factor(_vp(LU), npad, npad, npad * npad, batch, _vp(piv), _vp(info), _vp(work), s))
    iters, resid = ctypes.c_int32(0), ctypes.c_double(0.0)
    status = lib.bem_zlu_refine_solve(_vp(K), n, n * n, n, _vp(LU), npad, npad, npad * npad, batch, _vp(piv),
                                      _vp(work), _vp(B), _vp(X), _vp(R), npad, npad * nrhs, nrhs, 1e-12, 30,
                                      _vp(ts), _vp(norms), _vp(err), ctypes.byref(iters), ctypes.byref(resid), s)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    if status == _lib.BEM_ERR_NOT_CONVERGED:
        return  # flagged
    _lib.check(status)
    assert resid.value <= 1e-12 and iters.value >= 1
    for i in range(batch):
        x = X[i, :, :n].T.cpu().numpy()
        ref = np.linalg.solve(mats[i], rhs[i])
        assert np.max(np.linalg.norm(x - ref, axis=0) / np.linalg.norm(ref, axis=0)) < 1e-12, i


def test_fp64_engine_reports_its_residual(oracle_mod, default_oracle_gf, tmp_path):
    """The float64 engine's sweep (lid panels included) carries the worst
    relative residual of its solves, checked against the unfactored K."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.meshes import mesh_vertical_cylinder
    from test_gpu_mixed import _shared_table_gf
    hull = mesh_vertical_cylinder(length=8.0, radius=2.5, resolution=(3, 24, 8)).immersed_part()
    body = FloatingBody(hull, rigid_body_dofs(), lid_mesh=hull.generate_lid())
    res = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), precision="fp64",
                     max_batch=3).solve_frequencies(body, [0.6, 1.7, 2.9])
    assert 0.0 < res.stats["fp64_residual"] <= 1e-12
    assert res.stats["fp64_solve_iters"] >= 1


def _mixed_factors(n, batch, rng):
    import torch
    lib = _lib.load()
    npad = -(-n // 128) * 128
    mats = [_dominant(n, rng) for _ in range(batch)]
    K = torch.zeros((batch, n, n), dtype=torch.complex128, device="cuda")
    for i in range(batch):
        K[i].T[:, :] = torch.as_tensor(mats[i])
    nbytes = int(lib.bem_clu_workspace_bytes(npad, batch))
    work = torch.empty(nbytes + 1024, dtype=torch.uint8, device="cuda")
    wptr = (work.data_ptr() + 1023) // 1024 * 1024
    piv = torch.zeros((batch, npad), dtype=torch.int32, device="cuda")
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(lib.bem_clu_factor(_vp(K), n, n * n, n, npad, batch, _vp(piv), _vp(info), _vp(wptr), _vp(err),
                                  _lib.stream_ptr()))
    return mats, npad, work, wptr, piv, err


def test_bounded_wait_runs_out_and_the_stream_stays_usable():
    import torch
    lib = _lib.load()
    rng = np.random.default_rng(11)
    n, batch, nrhs = 500, 2, 3  # 4 block rows of 128 per matrix
    mats, npad, work, wptr, piv, err = _mixed_factors(n, batch, rng)
    rhs = [rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs)) for _ in range(batch)]
    B = torch.zeros((batch, nrhs, npad), dtype=torch.complex128, device="cuda")
    for i in range(batch):
        B[i, :, :n] = torch.as_tensor(rhs[i].T)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    s = _lib.stream_ptr()
    # block row 0 never publishes its flag: the waits of rows 1..3 give up after
    # 20000 polls (a few milliseconds) and report through err
    Bw = B.clone()
    _lib.check(lib.bem_clu_solve_bounded(_vp(wptr), npad, batch, _vp(piv), _vp(Bw), npad, npad * nrhs, nrhs,
                                         20000, 0, _vp(err), s))
    torch.cuda.synchronize()
    assert int(err.item()) == 1
    # the same stream, no flag withheld: a correct solve
    err.zero_()
    Bo = B.clone()
    _lib.check(lib.bem_clu_solve_bounded(_vp(wptr), npad, batch, _vp(piv), _vp(Bo), npad, npad * nrhs, nrhs,
                                         20000, -1, _vp(err), s))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    for i in range(batch):
        x = Bo[i, :, :n].T.cpu().numpy()
        ref = np.linalg.solve(mats[i], rhs[i])
        assert np.abs(x - ref).max() / np.abs(ref).max() < 5e-3  # float32 factors
    # and the engine-facing entry point on that stream
    Bb = B.clone()
    _lib.check(lib.bem_clu_solve(_vp(wptr), npad, batch, _vp(piv), _vp(Bb), npad, npad * nrhs, nrhs, _vp(err), s))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(Bb, Bo)


def test_bounded_wait_arguments_checked():
    import torch
    lib = _lib.load()
    buf = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    st = lib.bem_clu_solve_bounded(_vp(buf), 256, 1, _vp(buf), _vp(buf), 256, 256, 1, 0, -1, _vp(buf),
                                   _lib.stream_ptr())
    assert st == _lib.BEM_ERR_INVALID_ARGUMENT
    st = lib.bem_clu_solve_bounded(_vp(buf), 256, 1, _vp(buf), _vp(buf), 256, 256, 1, 100, 2, _vp(buf),
                                   _lib.stream_ptr())
    assert st == _lib.BEM_ERR_INVALID_ARGUMENT


def test_grouped_factorisation_equals_the_padded_one():
    """Matrices of different sizes in one padded batch: the grouped
    factorisation (tiles beyond each matrix's active size skipped) gives the
    factors of the plain batched one bit for bit, and solves each system."""
    import torch
    lib = _lib.load()
    rng = np.random.default_rng(21)
    npad, nrhs = 640, 2
    sizes = [250, 640, 380, 129]
    active = (ctypes.c_int32 * len(sizes))(*[-(-m // 128) * 128 for m in sizes])
    batch = len(sizes)
    K = torch.zeros((batch, npad, npad), dtype=torch.complex128, device="cuda")  # K[b].T column-major
    mats, rhs = [], []
    for b, m in enumerate(sizes):
        A = _dominant(m, rng)
        mats.append(A)
        K[b].T[:m, :m] = torch.as_tensor(A)
        K[b].T[m:, m:] = torch.eye(npad - m, dtype=torch.complex128)  # identity padding
        rhs.append(rng.standard_normal((m, nrhs)) + 1j * rng.standard_normal((m, nrhs)))
    B = torch.zeros((batch, nrhs, npad), dtype=torch.complex128, device="cuda")
    for b, m in enumerate(sizes):
        B[b, :, :m] = torch.as_tensor(rhs[b].T)
    s = _lib.stream_ptr()
    out = []
    for grouped in (False, True):
        nbytes = int(lib.bem_clu_workspace_bytes(npad, batch))
        work = torch.empty(nbytes + 1024, dtype=torch.uint8, device="cuda")
        wptr = (work.data_ptr() + 1023) // 1024 * 1024
        piv = torch.zeros((batch, npad), dtype=torch.int32, device="cuda")
        info = torch.zeros(batch, dtype=torch.int32, device="cuda")
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        if grouped:
            _lib.check(lib.bem_clu_factor_grouped(_vp(K), npad, npad * npad, npad, npad, batch, active, _vp(piv),
                                                  _vp(info), _vp(wptr), _vp(err), s))
        else:
            _lib.check(lib.bem_clu_factor(_vp(K), npad, npad * npad, npad, npad, batch, _vp(piv), _vp(info),
                                          _vp(wptr), _vp(err), s))
        X = B.clone()
        _lib.check(lib.bem_clu_solve(_vp(wptr), npad, batch, _vp(piv), _vp(X), npad, npad * nrhs, nrhs, _vp(err), s))
        torch.cuda.synchronize()
        assert int(err.item()) == 0 and info.cpu().numpy().tolist() == [0] * batch
        out.append(X)
    assert torch.equal(out[0], out[1])
    for b, m in enumerate(sizes):
        x = out[1][b, :, :m].T.cpu().numpy()
        ref = np.linalg.solve(mats[b], rhs[b])
        assert np.abs(x - ref).max() / np.abs(ref).max() < 5e-3
    bad = (ctypes.c_int32 * batch)(128, 100, 128, 128)  # not a multiple of 128
    assert lib.bem_clu_factor_grouped(_vp(K), npad, npad * npad, npad, npad, batch, bad, _vp(piv), _vp(info),
                                      _vp(wptr), _vp(err), s) == _lib.BEM_ERR_INVALID_ARGUMENT


def test_sweep_assembled_into_the_lu_planes_gives_the_same_factors(default_oracle_gf, tmp_path):
    """The frequency-sweep assembly that also writes K rounded to float32
    into the mixed LU's workspace (bem_assemble_wave_symmetric_batched_lu),
    factored by bem_clu_factor_planes, gives S, K and the factors of the
    plain sweep assembly followed by bem_clu_factor's conversion, bit for bit
    (npad > n, so the identity padding is written too)."""
    import torch
    from capytaine_b200.engine import B200Engine, _Factors
    from capytaine_b200.meshes import mesh_sphere
    from test_gpu_mixed import _shared_table_gf
    eng = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), precision="mixed")
    mesh = mesh_sphere(radius=1.0, resolution=(10, 30)).immersed_part()
    n = mesh.nb_faces
    assert n % 128 != 0
    ks = [0.3, 0.8, 1.7]
    out = []
    for planes in (True, False):
        f = _Factors(n, len(ks), "cuda", "mixed")
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        f.lu_work.zero_()
        eng.assemble_stage(f, mesh, ks, planes=planes)
        assert f.planes_ready == planes
        eng.factor_stage(f, len(ks), err)
        torch.cuda.synchronize()
        assert int(err.item()) == 0 and not f.planes_ready
        off = f.lu_work_ptr - f.lu_work.data_ptr()
        w_bytes = len(ks) * 2 * f.npad * f.npad * 4
        out.append((f.S.clone(), f.K.clone(), f.lu_work[off:off + w_bytes].clone(), f.info.clone()))
    for a, b in zip(out[0], out[1]):
        assert torch.equal(a, b)
