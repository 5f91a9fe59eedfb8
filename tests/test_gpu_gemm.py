"""The grouped FP64 DMMA GEMM (every autotuner variant) on single regular and
ragged problems through dmrgb200_dgemm_f64, against torch's FP64 matmul
(relative error <= 1e-13)."""
import ctypes as C

import pytest

from dmrgb200 import _capi as capi

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SHAPES = [(37, 53, 29, 0), (100, 7, 300, 3), (257, 129, 65, 1), (16, 64, 16, 0), (1, 1, 1, 0), (33, 65, 0, 0)]


@pytest.mark.parametrize("variant", range(capi.lib.dmrgb200_gemm_variant_count()))
@pytest.mark.parametrize("M,N,K,pad", SHAPES)
def test_dgemm_f64_matches_torch(variant, M, N, K, pad):
    assert torch.cuda.is_available()
    g = torch.Generator(device="cuda").manual_seed(M * 131 + N * 7 + K + variant)
    lda, ldb, ldc = M + pad, K + pad, M + 2 * pad
    A = torch.randn(max(K * lda, 1), dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(max(N * ldb, 1), dtype=torch.float64, device="cuda", generator=g)
    Cm = torch.full((N * ldc,), float("nan"), dtype=torch.float64, device="cuda")
    capi.check(capi.lib.dmrgb200_dgemm_f64(M, N, K, A.data_ptr(), lda, B.data_ptr(), ldb, Cm.data_ptr(), ldc,
                                           variant, None), "dgemm_f64")
    a = A[:K * lda].view(K, lda)[:, :M].T if K else torch.zeros(M, 0, dtype=torch.float64, device="cuda")
    b = B[:N * ldb].view(N, ldb)[:, :K].T if K else torch.zeros(0, N, dtype=torch.float64, device="cuda")
    ref = a @ b
    got = Cm.view(N, ldc)[:, :M].T
    err = (got - ref).norm() / max(ref.norm(), 1e-300)
    assert float(err) <= 1e-13 or (K == 0 and float(got.abs().max()) == 0.0)
    # the padding rows of C are not written
    if pad:
        assert torch.isnan(Cm.view(N, ldc)[:, M:]).all()
