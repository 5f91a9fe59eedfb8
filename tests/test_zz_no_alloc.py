"""dmrgb200_hpsi_noalloc: H·psi for callers that cannot allocate device memory.

Callers such as code running under a custom allocator or memory pool that owns
the device memory (and forbids further cudaMalloc), or hosts that only hand the
library pre-placed buffers, use the allocation-free entry point, which keeps its
tables and intermediates in a static device array.  This test calls it through
the C ABI twice in a row and checks both results against the regular entry
point dmrgb200_hpsi (same FP64 tolerance as the parity tests).  Runs last so
that a failure here comes after every other test; it passes on its own too.
"""
import ctypes as C

import numpy as np
import pytest

from dmrgb200 import _capi as capi
from dmrgb200 import engine as E
from helpers import OracleChain, make_chain, random_psi

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12


def test_noalloc_matches_hpsi_twice():
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    ctx = E.Context(0)
    model, bonds, tensors, rng = make_chain("hubbard", 12, 0, seed=17, synthetic_m=64)
    ch = OracleChain(model, bonds, tensors, 5)
    Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
    la, ra = ch.Lidx.cohort_addresses(Lb.data_ptr()), ch.Ridx.cohort_addresses(Rb.data_ptr())
    plan = E.DevicePlan(ctx, ch.sched.plan, left_addr=la, other_addr=ra)
    desc, keep = capi.numpy_to_desc(ch.sched.plan)
    lv, larr = E._view(la)
    rv, rarr = E._view(ra)
    for call in range(2):
        x = E.to_device(random_psi(ch.p12, ch.left, ch.right, rng).data)
        y_ref = torch.zeros_like(x)
        y = torch.full_like(x, float("nan")) if call == 0 else torch.zeros_like(x)
        plan.hpsi(x.data_ptr(), y_ref.data_ptr())
        torch.cuda.synchronize()
        # the first call on the device may place the static array (lazy module
        # loading); the second must leave the device's free memory and torch's
        # allocations exactly as they were
        free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
        st = capi.lib.dmrgb200_hpsi_noalloc(C.byref(desc), C.byref(lv), C.byref(rv), x.data_ptr(), y.data_ptr(), None)
        capi.check(st, "dmrgb200_hpsi_noalloc")
        torch.cuda.synchronize()
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free0, "the call changed the device's free memory"
            assert torch.cuda.memory_allocated() == alloc0
        a, b = y.cpu().numpy(), y_ref.cpu().numpy()
        mask = np.zeros(a.shape, dtype=bool)
        for off, r, c in zip(ch.sched.plan["out_off"], ch.sched.plan["out_rows"], ch.sched.plan["out_cols"]):
            mask[int(off):int(off) + int(r) * int(c)] = True
        err = np.linalg.norm(a[mask] - b[mask]) / np.linalg.norm(b[mask])
        assert err <= TOL, (call, err)
    del keep, larr, rarr


def test_noalloc_rejects_a_plan_beyond_the_static_area():
    """A plan whose T intermediate alone is 64 MiB returns DMRGB200_OUT_OF_MEMORY
    with the required size, and the next call on a fitting plan still succeeds."""
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from test_capi_errors import one_task_plan

    big = one_task_plan(ls=1024, rs=1024, nb=8)
    desc, keep = capi.numpy_to_desc(big)
    xb = torch.zeros(big["in_size"], dtype=torch.float64, device="cuda")
    yb = torch.zeros_like(xb)
    Rb = torch.zeros(8 * 1024 * 1024, dtype=torch.float64, device="cuda")
    Lb = torch.zeros(1024 * 1024, dtype=torch.float64, device="cuda")
    lv, larr = E._view([Lb.data_ptr()])
    rv, rarr = E._view([Rb.data_ptr()])
    st = capi.lib.dmrgb200_hpsi_noalloc(C.byref(desc), C.byref(lv), C.byref(rv), xb.data_ptr(), yb.data_ptr(), None)
    msg = capi.lib.dmrgb200_last_error().decode()
    assert st == 3 and "bytes of scratch" in msg, (st, msg)
    small = one_task_plan(ls=8, rs=8, nb=2)
    desc2, keep2 = capi.numpy_to_desc(small)
    xs = torch.rand(64, dtype=torch.float64, device="cuda")
    ys = torch.zeros_like(xs)
    R2 = torch.rand(2 * 64, dtype=torch.float64, device="cuda")
    L2 = torch.rand(64, dtype=torch.float64, device="cuda")
    lv2, la2 = E._view([L2.data_ptr()])
    rv2, ra2 = E._view([R2.data_ptr()])
    capi.check(capi.lib.dmrgb200_hpsi_noalloc(C.byref(desc2), C.byref(lv2), C.byref(rv2), xs.data_ptr(),
                                              ys.data_ptr(), None), "dmrgb200_hpsi_noalloc")
    # y = L^T-free check: one term, alpha 1, b1 = 0: y = L_0 (8x8) * (x (8x8) * R_0 (8x8))
    X = xs.view(8, 8).T
    Y = L2.view(8, 8).T @ (X @ R2[:64].view(8, 8).T)
    got = ys.view(8, 8).T
    assert torch.allclose(got, Y, rtol=1e-12, atol=1e-12), float((got - Y).abs().max())
    del keep, keep2, larr, rarr, la2, ra2
