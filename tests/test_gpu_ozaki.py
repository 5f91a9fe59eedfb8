"""FP64 GEMM emulated on the INT8 tensor cores (dmrgb200_dgemm_emulated)
against numpy FP64: the relative error falls like 2^(-7 slices) of the row and
column maxima."""
import ctypes as C

import numpy as np
import pytest

from dmrgb200 import _capi as capi

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _emulated(A, B, slices):
    M, K = A.shape
    N = B.shape[1]
    # column-major storage: torch tensors hold the transposed (row-major) view
    Ad = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    Bd = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    Cd = torch.zeros((N, M), dtype=torch.float64, device="cuda")
    st = capi.lib.dmrgb200_dgemm_emulated(M, N, K, Ad.data_ptr(), M, Bd.data_ptr(), K, Cd.data_ptr(), M, slices,
                                          None)
    capi.check(st, "dmrgb200_dgemm_emulated")
    torch.cuda.synchronize()
    return Cd.cpu().numpy().T


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (128, 64, 192), (256, 128, 64), (300, 200, 500), (37, 5, 11)])
def test_emulated_gemm_accuracy(M, N, K):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    A = rng.standard_normal((M, K)) * np.exp(rng.uniform(-3, 3, (M, 1)))
    B = rng.standard_normal((K, N)) * np.exp(rng.uniform(-3, 3, (1, N)))
    ref = A @ B
    scale = np.abs(A).max(axis=1)[:, None] * np.abs(B).max(axis=0)[None, :] * K
    for s, tol in [(7, 1e-14), (5, 1e-10), (3, 1e-5)]:
        got = _emulated(A, B, s)
        err = np.max(np.abs(got - ref) / scale)
        assert err <= tol, (s, err)


def test_emulated_gemm_rejects_bad_arguments():
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    assert capi.lib.dmrgb200_dgemm_emulated(4, 4, 4, d.data_ptr(), 4, d.data_ptr(), 4, d.data_ptr(), 4, 9,
                                            None) == 1
    assert capi.lib.dmrgb200_dgemm_emulated(4, 4, 4, d.data_ptr(), 3, d.data_ptr(), 4, d.data_ptr(), 4, 7,
                                            None) == 1


@pytest.mark.parametrize("s,K", [(7, 40000), (8, 16384 + 64), (3, 2 * 43648 + 5)])
def test_emulated_gemm_long_k_in_chunks(s, K):
    """K beyond 2^17 / slices: the tile accumulates exact INT32 chunks of
    floor(2^17 / (64 s)) slabs of 64 and adds each chunk's FP64 partial product
    into C; the error bound stays that of the split."""
    M, N = 130, 70
    rng = np.random.default_rng(K + s)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((K, N))
    ref = A @ B
    scale = np.abs(A).max(axis=1)[:, None] * np.abs(B).max(axis=0)[None, :] * K
    tol = {7: 1e-14, 8: 1e-14, 3: 1e-5}[s]
    err = np.max(np.abs(_emulated(A, B, s) - ref) / scale)
    assert err <= tol, err
