"""The drop-in seam on the device: a schedule held in the reference's own
ScheduleNew objects is flattened by the reference-side flattener
(oracle/ref_flatten.cpp) and handed to dmrgb200_plan_create; the device H·psi of
that plan matches the reference's own CPU execution of the ScheduleNew
(tasks.cpp create_T / contract) and is bitwise that of the library's own plan."""
import numpy as np
import pytest

import ref as REF
from dmrgb200 import engine as E
from helpers import OracleChain, make_chain, random_psi

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not REF.available(), reason="oracle/_ref not built (reference sources absent)")]


@pytest.mark.parametrize("name,L,m", [("hubbard", 12, 64), ("qc", 8, 48)])
def test_flattened_reference_schedule_runs_on_the_device(name, L, m):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    ctx = E.Context(0)
    model, bonds, tensors, rng = make_chain(name, L, 0, seed=8, synthetic_m=m)
    ch = OracleChain(model, bonds, tensors, L // 2 - 1)
    h = REF.Hpsi(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx)
    flat = h.flatten()
    Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
    la, ra = ch.Lidx.cohort_addresses(Lb.data_ptr()), ch.Ridx.cohort_addresses(Rb.data_ptr())
    plan_ref = E.DevicePlan(ctx, flat, left_addr=la, other_addr=ra)
    plan_own = E.DevicePlan(ctx, ch.sched.plan, left_addr=la, other_addr=ra)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    xd = E.to_device(x)
    y1, y2 = torch.zeros_like(xd), torch.zeros_like(xd)
    plan_ref.hpsi(xd.data_ptr(), y1.data_ptr())
    plan_own.hpsi(xd.data_ptr(), y2.data_ptr())
    torch.cuda.synchronize()
    a, b = y1.cpu().numpy(), y2.cpu().numpy()
    assert np.array_equal(a, b)
    yref = h.run(x)
    assert np.linalg.norm(a - yref) <= 1e-12 * np.linalg.norm(yref)
