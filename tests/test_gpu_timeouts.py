"""Failure detection of the device-side waits, without faulting the GPU: the limit
of the bounded waits for pipeline data (dmrgb200_set_wait_limit) is set to 1 ns,
so the grouped S build's and the emulated stages' waits for their bulk copies run
out; the kernels record it in the plan's error words, let their in-flight copies
and MMAs complete under the fixed 2 s limit, release their tensor memory and
return.  The host then sees DMRGB200_TIMEOUT from dmrgb200_plan_check (and from a
stepwise dmrgb200_solve), and, with the default limit restored, the next call on
the same plan succeeds and matches the oracle."""
import numpy as np
import pytest

from dmrgb200 import _capi as capi
from dmrgb200 import engine as E
from helpers import OracleChain, make_chain, random_psi

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TIMEOUT = 5


@pytest.fixture
def grouped_plan(monkeypatch):
    """A quantum-chemistry H·psi plan whose S build runs as line groups on bulk-copy rings."""
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    monkeypatch.setenv("DMRGB200_SBUILD", "groups")
    ctx = E.Context(0)
    model, bonds, tensors, rng = make_chain("qc", 8, 0, seed=6, synthetic_m=64)
    ch = OracleChain(model, bonds, tensors, 3)
    Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
    plan = E.DevicePlan(ctx, ch.sched.plan, left_addr=ch.Lidx.cohort_addresses(Lb.data_ptr()),
                        other_addr=ch.Ridx.cohort_addresses(Rb.data_ptr()))
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    yield plan, ch, x, (ctx, Lb, Rb)
    capi.lib.dmrgb200_set_wait_limit(0)


def _timed_out_once(plan, xd, yd, prec, tries=5):
    """Run H·psi under the 1 ns limit until a wait runs out (the first wait of a ring
    almost always does); True when dmrgb200_plan_check reported DMRGB200_TIMEOUT."""
    capi.check(capi.lib.dmrgb200_set_wait_limit(1), "set_wait_limit")
    try:
        for _ in range(tries):
            plan.hpsi(xd.data_ptr(), yd.data_ptr(), prec)
            try:
                plan.check()
            except capi.DmrgError as exc:
                assert exc.status == TIMEOUT, exc
                return True
        return False
    finally:
        capi.check(capi.lib.dmrgb200_set_wait_limit(0), "set_wait_limit")


@pytest.mark.parametrize("prec", [capi.PREC_FP64, capi.PREC_FP64_EMULATED])
def test_wait_timeout_is_reported_and_the_plan_recovers(grouped_plan, prec):
    plan, ch, x, _ = grouped_plan
    xd = E.to_device(x)
    yd = torch.zeros_like(xd)
    if prec == capi.PREC_FP64_EMULATED:
        plan.hpsi(xd.data_ptr(), yd.data_ptr(), prec)  # tables and boundary digit planes first
        plan.check()
    assert _timed_out_once(plan, xd, yd, prec)
    # default limit again: the same plan computes the right answer
    yd.zero_()
    plan.hpsi(xd.data_ptr(), yd.data_ptr(), prec)
    plan.check()
    ref = ch.hpsi(x)
    y = yd.cpu().numpy()
    err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
    assert err <= (1e-12 if prec == capi.PREC_FP64 else 1e-10), err


def test_stepwise_solve_reports_a_timeout(grouped_plan):
    plan, ch, x, _ = grouped_plan
    xd = E.to_device(x / np.linalg.norm(x))
    xo = torch.zeros_like(xd)
    plan.set_solver(capi.SOLVER_STEPWISE)
    capi.check(capi.lib.dmrgb200_set_wait_limit(1), "set_wait_limit")
    got = None
    try:
        for _ in range(5):
            try:
                plan.solve(xd.data_ptr(), xo.data_ptr(), xd.numel(), tol=0.0, max_iter=4)
            except capi.DmrgError as exc:
                got = exc.status
                break
    finally:
        capi.check(capi.lib.dmrgb200_set_wait_limit(0), "set_wait_limit")
    assert got == TIMEOUT
    e, st = plan.solve(xd.data_ptr(), xo.data_ptr(), xd.numel(), tol=0.0, max_iter=4)
    assert st.iterations == 4 and np.isfinite(e)
