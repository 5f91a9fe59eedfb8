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


def test_dumped_site_problem_runs_bitwise_the_same(tmp_path):
    """A site problem written by dmrgb200.dump and read back gives bitwise the
    device H·psi of the original plan."""
    from dmrgb200 import dump
    ctx = E.Context(0)
    model, bonds, tensors, rng = make_chain("hubbard", 12, 0, seed=9, synthetic_m=64)
    ch = OracleChain(model, bonds, tensors, 5)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    path = tmp_path / "site.npz"
    dump.save_site_problem(path, ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, psi=x)
    d = dump.load_site_problem(path)
    out = []
    for plan_d, L, Li, R, Ri, xx in ((ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, x),
                                     (d.plan, d.L, d.Lidx, d.R, d.Ridx, d.psi)):
        Lb, Rb = E.to_device(L), E.to_device(R)
        plan = E.DevicePlan(ctx, plan_d, left_addr=Li.cohort_addresses(Lb.data_ptr()),
                            other_addr=Ri.cohort_addresses(Rb.data_ptr()))
        xd = E.to_device(xx)
        yd = torch.zeros_like(xd)
        plan.hpsi(xd.data_ptr(), yd.data_ptr())
        torch.cuda.synchronize()
        out.append(yd.cpu().numpy())
    assert np.array_equal(out[0], out[1])


def test_plan_reuse_across_sweeps():
    """Sweeps with the backend's plan cache give the same energies as sweeps that
    rebuild every schedule and plan, and once the bond dimensions settle every
    site problem and boundary step is served from the cache."""
    from dmrgb200 import dmrg as G
    from dmrgb200 import models as M
    from dmrgb200 import mps as S
    ctx = E.Context(0)
    L = 10
    model = M.heisenberg(L)
    A = S.random_mps(model.phys, S.allowed_sectors(model.phys, L, model.total_charge, 5), np.random.default_rng(1))
    runs = {}
    for reuse in (False, True):
        be = G.DeviceBackend(ctx, reuse_plans=reuse)
        dm = G.TwoSiteDMRG(be, model, list(A), 32, jd_tol=1e-10, jd_maxiter=16)
        for sw in range(4):
            dm.sweep(sw)
        runs[reuse] = (np.array([e[2] for e in dm.log.energies]), be.cache_hits, be.cache_misses)
    assert np.abs(runs[True][0] - runs[False][0]).max() <= 1e-12
    hits, misses = runs[True][1], runs[True][2]
    assert hits >= 2 * (L - 1) * 2, (hits, misses)  # at least the last sweep's solves and steps
