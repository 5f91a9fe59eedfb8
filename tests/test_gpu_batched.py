"""Batched multi-instance H·psi: independent site problems (mixed U1 and TwoU1,
different bond dimensions) merged into one plan give, per instance, the oracle's
H·psi of that instance (FP64, relative error <= 1e-12)."""
import numpy as np
import pytest

from dmrgb200 import engine as E
from helpers import OracleChain, make_chain, random_psi

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_batched_instances_match_oracle():
    ctx = E.Context(0)
    specs = [("hubbard", 10, 40, 1), ("heisenberg", 16, 48, 2), ("hubbard", 12, 64, 3), ("bose", 10, 24, 4),
             ("heisenberg", 12, 16, 5)]
    chains, xs, keep = [], [], []
    for name, L, m, seed in specs:
        model, bonds, tensors, rng = make_chain(name, L, 0, seed=seed, synthetic_m=m)
        ch = OracleChain(model, bonds, tensors, L // 2 - 1)
        Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
        keep += [Lb, Rb]
        chains.append((ch, ch.Lidx.cohort_addresses(Lb.data_ptr()), ch.Ridx.cohort_addresses(Rb.data_ptr())))
        xs.append(random_psi(ch.p12, ch.left, ch.right, rng).data)
    bp = E.BatchedPlan(ctx, [(c.sched.plan, la, ra) for c, la, ra in chains])
    x = np.zeros(bp.total_size)
    for b, xi in zip(bp.in_base, xs):
        x[b:b + xi.size] = xi
    xd = E.to_device(x)
    yd = torch.zeros_like(xd)
    bp.hpsi(xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    y = yd.cpu().numpy()
    assert bp.flops == sum(c.sched.flops for c, _, _ in chains)
    for (c, _, _), b, xi in zip(chains, bp.in_base, xs):
        ref = c.hpsi(xi)
        got = y[b:b + xi.size]
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
