"""The allocation-free entry point bem_zgemm_ts_static, for callers that can
only pass buffers they already own (no device allocation of their own), must
give the same result as bem_zgemm_ts with a caller workspace, and must not
take device memory of its own once the library is loaded.

Two calls in a row share the library's static scratch array: the second call
(different sizes, beta != 0) must not see anything left by the first.  The
file name sorts after every other test file, so pytest collects it last; it
needs no other test."""
import ctypes

import numpy as np
import pytest

from capytaine_b200 import _lib

pytestmark = pytest.mark.gpu

RTOL = 1e-13  # same bar as the other split-K GEMM tests


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _case(M, K, nrhs, batch, seed):
    import torch
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((batch, M, K)) + 1j * rng.standard_normal((batch, M, K))
    x = rng.standard_normal((batch, K, nrhs)) + 1j * rng.standard_normal((batch, K, nrhs))
    y = rng.standard_normal((batch, M, nrhs)) + 1j * rng.standard_normal((batch, M, nrhs))
    # column-major per batch entry: element (i, j) at i + j*ld
    At = torch.as_tensor(np.ascontiguousarray(a.transpose(0, 2, 1)), device="cuda")
    Xt = torch.as_tensor(np.ascontiguousarray(x.transpose(0, 2, 1)), device="cuda")
    Yt = torch.as_tensor(np.ascontiguousarray(y.transpose(0, 2, 1)), device="cuda")
    return At, Xt, Yt


def _run(static, At, Xt, Yt, M, K, nrhs, batch, alpha, beta):
    import torch
    lib = _lib.load()
    Y = Yt.clone()
    args = (M, K, nrhs, alpha.real, alpha.imag, _vp(At), M, M * K, _vp(Xt), K, K * nrhs, beta.real, beta.imag,
            _vp(Y), M, M * nrhs, batch)
    if static:
        _lib.check(lib.bem_zgemm_ts_static(*args, _lib.stream_ptr()))
    else:
        work = torch.empty(int(lib.bem_zgemm_ts_workspace_bytes(M, K, nrhs, batch)), dtype=torch.uint8,
                           device="cuda")
        _lib.check(lib.bem_zgemm_ts(*args, _vp(work), _lib.stream_ptr()))
    torch.cuda.synchronize()
    return Y.cpu().numpy()


def test_static_scratch_variant_matches_workspace_variant_twice():
    lib = _lib.load()
    assert lib.bem_zgemm_ts_static_capacity() == 1 << 19
    calls = [
        # (M, K, nrhs, batch, alpha, beta): 6084-panel S @ sigma shape, then a second,
        # different call accumulating into Y
        (6084, 6084, 7, 1, 1.0 + 0.0j, 0.0 + 0.0j),
        (1000, 3000, 16, 3, 0.5 - 2.0j, 1.0 + 1.0j),
    ]
    for i, (M, K, nrhs, batch, alpha, beta) in enumerate(calls):
        At, Xt, Yt = _case(M, K, nrhs, batch, seed=i)
        ref = _run(False, At, Xt, Yt, M, K, nrhs, batch, alpha, beta)
        got = _run(True, At, Xt, Yt, M, K, nrhs, batch, alpha, beta)
        assert np.abs(got - ref).max() / np.abs(ref).max() < RTOL, i


def test_static_call_takes_no_device_memory():
    """Free device memory (cudaMemGetInfo) is the same before and after a
    static call made once the first call has looked the array up."""
    import torch
    lib = _lib.load()
    M, K, nrhs, batch = 3000, 2000, 8, 2
    At, Xt, Yt = _case(M, K, nrhs, batch, seed=7)
    args = (M, K, nrhs, 1.0, 0.0, _vp(At), M, M * K, _vp(Xt), K, K * nrhs, 0.0, 0.0, _vp(Yt), M, M * nrhs, batch,
            _lib.stream_ptr())
    _lib.check(lib.bem_zgemm_ts_static(*args))
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    _lib.check(lib.bem_zgemm_ts_static(*args))
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before


def test_static_scratch_batch_limit():
    import torch
    lib = _lib.load()
    A = torch.zeros((4, 4), dtype=torch.complex128, device="cuda")
    status = lib.bem_zgemm_ts_static(1, 4, 1, 1.0, 0.0, _vp(A), 1, 0, _vp(A), 4, 0, 0.0, 0.0, _vp(A), 1, 0, 70000,
                                     _lib.stream_ptr())
    assert status == _lib.BEM_ERR_INVALID_ARGUMENT
    assert b"65535" in lib.bem_last_error()


def test_static_scratch_capacity_is_enforced():
    import torch
    lib = _lib.load()
    M, K, nrhs = 40000, 64, 16  # M * nrhs > capacity
    A = torch.zeros((K, M), dtype=torch.complex128, device="cuda")
    X = torch.zeros((nrhs, K), dtype=torch.complex128, device="cuda")
    Y = torch.zeros((nrhs, M), dtype=torch.complex128, device="cuda")
    status = lib.bem_zgemm_ts_static(M, K, nrhs, 1.0, 0.0, _vp(A), M, 0, _vp(X), K, 0, 0.0, 0.0, _vp(Y), M, 0, 1,
                                     _lib.stream_ptr())
    assert status == _lib.BEM_ERR_INVALID_ARGUMENT
    assert b"static scratch capacity" in lib.bem_last_error()
