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
        st = capi.lib.dmrgb200_hpsi_noalloc(C.byref(desc), C.byref(lv), C.byref(rv), x.data_ptr(), y.data_ptr(), None)
        capi.check(st, "dmrgb200_hpsi_noalloc")
        torch.cuda.synchronize()
        a, b = y.cpu().numpy(), y_ref.cpu().numpy()
        mask = np.zeros(a.shape, dtype=bool)
        for off, r, c in zip(ch.sched.plan["out_off"], ch.sched.plan["out_rows"], ch.sched.plan["out_cols"]):
            mask[int(off):int(off) + int(r) * int(c)] = True
        err = np.linalg.norm(a[mask] - b[mask]) / np.linalg.norm(b[mask])
        assert err <= TOL, (call, err)
    del keep, larr, rarr
