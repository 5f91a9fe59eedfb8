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


def test_pinned_plan_variants_match_oracle():
    """dmrgb200_plan_set_gemm_variants: every variant pinned on both stages of an H·psi plan
    gives the oracle's H·psi (FP64, 1e-12), on the device and through the host-buffer graph
    (which is captured again after a new choice); an index out of range is rejected."""
    import numpy as np

    from dmrgb200 import engine as E
    from helpers import OracleChain, make_chain, random_psi

    model, bonds, tensors, rng = make_chain("qc", 8, 0, seed=5, synthetic_m=64)
    ch = OracleChain(model, bonds, tensors, 3)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    want = ch.hpsi(x)
    ctx = E.Context(0)
    Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
    plan = E.DevicePlan(ctx, ch.sched.plan, left_addr=ch.Lidx.cohort_addresses(Lb.data_ptr()),
                        other_addr=ch.Ridx.cohort_addresses(Rb.data_ptr()))
    xd = E.to_device(x)
    xh = torch.tensor(x, dtype=torch.float64).pin_memory()
    yh = torch.zeros(len(want), dtype=torch.float64).pin_memory()
    n = capi.lib.dmrgb200_gemm_variant_count()
    for v in range(n):
        plan.set_gemm_variants(v, (v + 3) % n)
        yd = torch.zeros_like(xd)
        plan.hpsi(xd.data_ptr(), yd.data_ptr())
        plan.hpsi_host(xh.data_ptr(), yh.data_ptr())
        torch.cuda.synchronize()
        for got in (yd.cpu().numpy(), yh.numpy()):
            assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want), v
    with pytest.raises(capi.DmrgError) as e:
        plan.set_gemm_variants(n, 0)
    assert e.value.status == capi.INVALID_ARGUMENT
