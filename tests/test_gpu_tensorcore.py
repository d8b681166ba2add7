"""tcgen05 TF32 complex update against NumPy (complex128 reference).  TF32
keeps 10 mantissa bits: the error bar is 2e-3 of |A| |B| summed over K."""
import ctypes

import numpy as np
import pytest

from capytaine_b200 import _lib

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def pack_a(A):
    """rows i: [Re A(i,:), Im A(i,:)]"""
    return np.concatenate([A.real, A.imag], axis=1).astype(np.float32)


def pack_b(B):
    """per 128-column group: 128 rows [Re; -Im] then 128 rows [Im; Re]."""
    k, n = B.shape
    out = np.zeros((2 * n, 2 * k), dtype=np.float32)
    for j0 in range(0, n, 128):
        blk = B[:, j0:j0 + 128]
        out[2 * j0: 2 * j0 + 128] = np.concatenate([blk.real, -blk.imag], axis=0).T
        out[2 * j0 + 128: 2 * j0 + 256] = np.concatenate([blk.imag, blk.real], axis=0).T
    return out


# the last case has 512 tiles of 128 x 128: more than one per SM, so each CTA of
# the persistent kernel alternates between its two tensor-memory accumulators
@pytest.mark.parametrize("m,n,k,batch", [(128, 128, 16, 1), (256, 384, 64, 2), (512, 256, 128, 1),
                                         (2048, 2048, 64, 2)])
def test_cgemm_tf32_update(m, n, k, batch):
    import torch
    rng = np.random.default_rng(m + n + k)
    lib = _lib.load()
    A = [rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k)) for _ in range(batch)]
    B = [rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n)) for _ in range(batch)]
    C = [rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n)) for _ in range(batch)]
    # operands of shape [batch][rows][2k]; C planes column-major with an offset block
    r0, c0 = 64, 128
    ldc = r0 + m + 32
    ncols = c0 + n
    Aop = torch.as_tensor(np.stack([pack_a(a) for a in A]), device="cuda")
    Bop = torch.as_tensor(np.stack([pack_b(b) for b in B]), device="cuda")
    Cr = torch.zeros((batch, ncols, ldc), dtype=torch.float32, device="cuda")
    Ci = torch.zeros_like(Cr)
    for b in range(batch):
        Cr[b, c0:, r0:r0 + m] = torch.as_tensor(C[b].real.T.astype(np.float32))
        Ci[b, c0:, r0:r0 + m] = torch.as_tensor(C[b].imag.T.astype(np.float32))
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(lib.bem_cgemm_tf32_update(_vp(Aop), m, 0, _vp(Bop), 2 * n, 0, 2 * k, _vp(Cr), _vp(Ci), ldc,
                                         ncols * ldc, r0, c0, m, n, batch, _vp(err), _lib.stream_ptr()))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    for b in range(batch):
        got = Cr[b, c0:, r0:r0 + m].cpu().numpy().T + 1j * Ci[b, c0:, r0:r0 + m].cpu().numpy().T
        ref = C[b].astype(np.complex64).astype(np.complex128) - A[b] @ B[b]
        scale = np.abs(A[b]) @ np.abs(B[b])
        assert np.max(np.abs(got - ref) / (scale + 1e-30)) < 2e-3
        # entries outside the block are untouched
        assert float(Cr[b, :c0].abs().max()) == 0.0 and float(Cr[b, c0:, :r0].abs().max()) == 0.0
