"""Jacobi-Davidson on a batched plan (dmrgb200.batched.BatchedJD): every instance's
energy after the same number of iterations equals the oracle JD (numpy
restatement of ietl/jacobi.h) on that instance alone, and the emulated batched
solve stays within 1e-9 of the FP64 one per instance."""
import numpy as np
import pytest

import jd as JD
import oracle as O
from dmrgb200 import _capi as capi
from dmrgb200 import batched as B
from dmrgb200 import dmrg as G
from dmrgb200 import engine as E
from dmrgb200 import models as M
from dmrgb200 import mps as S

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_batched_jd_matches_per_instance_oracle():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    ctx = E.Context(0)
    rng = np.random.default_rng(6)
    sps, items = [], []
    for k in range(6):
        L = 12
        model = M.heisenberg(L) if k % 2 == 0 else M.fermi_hubbard(L)
        m = int(rng.integers(16, 48))
        bonds = S.synthetic_bonds(model.phys, L, model.total_charge, m, 10.0 if k % 2 == 0 else 3.5)
        i = L // 2 - 1
        A = G.left_canonicalize(G.right_canonicalize(S.random_mps(model.phys, bonds, rng), 0.0), i, 0.0)
        bonds = [t.left for t in A] + [A[-1].right]
        sp = E.SiteProblem(ctx, model, A, bonds, i)
        sps.append(sp)
        items.append((sp.schedule.plan, sp.Lidx.cohort_addresses(sp.Lbuf.data_ptr()),
                      sp.Ridx.cohort_addresses(sp.Rbuf.data_ptr())))
    bp = E.BatchedPlan(ctx, items)
    x0 = torch.zeros(bp.total_size, dtype=torch.float64, device="cuda")
    starts = []
    for sp, b in zip(sps, bp.in_base):
        x = np.zeros(sp.size)
        pl = sp.schedule.plan
        for off, r, c in zip(pl["in_off"], pl["in_rows"], pl["in_cols"]):
            x[int(off):int(off) + int(r) * int(c)] = rng.standard_normal(int(r) * int(c))
        x /= np.linalg.norm(x)
        starts.append(x)
        x0[b:b + sp.size] = torch.from_numpy(x)
    solver = B.BatchedJD(bp)
    th64, u64, it64, _ = solver.solve(x0, max_iter=10)
    them, _, _, _ = solver.solve(x0, max_iter=10, prec=capi.PREC_FP64_EMULATED)
    th64, them = th64.cpu().numpy(), them.cpu().numpy()
    assert (it64.cpu().numpy() == 10).all()
    for k, sp in enumerate(sps):
        Lv, Rv = sp.Lbuf.cpu().numpy(), sp.Rbuf.cpu().numpy()
        pl = sp.schedule.plan
        theta, _, _, _, _ = JD.jcd(lambda v: O.hpsi(pl, Lv, sp.Lidx, Rv, sp.Ridx, v), starts[k], tol=0.0, max_iter=10)
        assert abs(th64[k] - theta) <= 1e-10 * max(1.0, abs(theta)), (k, th64[k], theta)
        assert abs(them[k] - th64[k]) <= 1e-9 * max(1.0, abs(theta)), (k, them[k], th64[k])
