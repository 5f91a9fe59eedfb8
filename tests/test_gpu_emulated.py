"""H·psi with the contractions emulated on the INT8 tensor cores
(DMRGB200_PREC_FP64_EMULATED) against the oracle: relative error per H·psi
<= 1e-10 with 6 digit planes and <= 1e-12 with 7."""
import ctypes as C

import numpy as np
import pytest

from dmrgb200 import _capi as capi
from dmrgb200 import engine as E
from helpers import OracleChain, make_chain, random_psi

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,L,m", [("hubbard", 12, 64), ("heisenberg", 16, 48), ("bose", 10, 32)])
def test_emulated_hpsi_matches_oracle(name, L, m):
    ctx = E.Context(0)
    model, bonds, tensors, rng = make_chain(name, L, 0, seed=3, synthetic_m=m)
    ch = OracleChain(model, bonds, tensors, L // 2 - 1)
    Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
    plan = E.DevicePlan(ctx, ch.sched.plan, left_addr=ch.Lidx.cohort_addresses(Lb.data_ptr()),
                        other_addr=ch.Ridx.cohort_addresses(Rb.data_ptr()))
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    ref = ch.hpsi(x)
    xd = E.to_device(x)
    for slices, tol in [(7, 1e-12), (6, 1e-10)]:
        capi.check(capi.lib.dmrgb200_plan_set_slices(plan.handle, slices), "set_slices")
        yd = torch.full_like(xd, float("nan"))
        mask = torch.zeros_like(xd, dtype=torch.bool)
        for off, r, c in zip(ch.sched.plan["out_off"], ch.sched.plan["out_rows"], ch.sched.plan["out_cols"]):
            mask[int(off):int(off) + int(r) * int(c)] = True
        yd[~mask] = 0.0
        plan.hpsi(xd.data_ptr(), yd.data_ptr(), capi.PREC_FP64_EMULATED)
        torch.cuda.synchronize()
        y = yd.cpu().numpy()
        err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
        assert err <= tol, (slices, err)


def test_emulated_reuses_boundary_digits_across_calls():
    """The boundaries' digit planes are made on the first emulated call and reused:
    three calls with different vectors each match the oracle, and repeating the
    first vector reproduces its result bitwise."""
    ctx = E.Context(0)
    model, bonds, tensors, rng = make_chain("hubbard", 12, 0, seed=8, synthetic_m=64)
    ch = OracleChain(model, bonds, tensors, 5)
    Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
    plan = E.DevicePlan(ctx, ch.sched.plan, left_addr=ch.Lidx.cohort_addresses(Lb.data_ptr()),
                        other_addr=ch.Ridx.cohort_addresses(Rb.data_ptr()))
    capi.check(capi.lib.dmrgb200_plan_set_slices(plan.handle, 7), "set_slices")
    xs = [random_psi(ch.p12, ch.left, ch.right, rng).data for _ in range(2)]
    outs = []
    for x in (xs[0], xs[1], xs[0]):
        xd = E.to_device(x)
        yd = torch.zeros_like(xd)
        plan.hpsi(xd.data_ptr(), yd.data_ptr(), capi.PREC_FP64_EMULATED)
        torch.cuda.synchronize()
        y = yd.cpu().numpy()
        ref = ch.hpsi(x)
        assert np.linalg.norm(y - ref) <= 1e-12 * np.linalg.norm(ref)
        outs.append(y)
    assert np.array_equal(outs[0], outs[2])
