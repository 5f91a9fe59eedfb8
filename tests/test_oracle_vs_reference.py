"""Pin of the oracle: its restatement of the reference's schedule execution
agrees with the reference's own solver core (tasks.cpp compiled from the
reference sources into oracle/_ref by oracle/build_ref.sh) on identical plans
and inputs, for H·psi and both boundary steps."""
import numpy as np
import pytest

import oracle as O
import ref as REF
from dmrgb200 import engine as E
from dmrgb200 import models as M
from helpers import OracleChain, make_chain, random_psi

pytestmark = pytest.mark.skipif(not REF.available(), reason="oracle/_ref not built (reference sources absent)")


@pytest.mark.parametrize("name,L,m", [("heisenberg", 12, 24), ("hubbard", 10, 40), ("bose", 10, 24)])
def test_hpsi_and_steps_match_reference_code(name, L, m):
    model, bonds, tensors, rng = make_chain(name, L, 0, seed=5, synthetic_m=m)
    i = L // 2 - 1
    ch = OracleChain(model, bonds, tensors, i)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    y_ours = O.hpsi(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, x)
    y_ref = REF.hpsi(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, x)
    assert np.linalg.norm(y_ours - y_ref) <= 1e-14 * np.linalg.norm(y_ref)
    # one left and one right step from the chain's boundaries
    t = tensors[i]
    W = M.MPOHandle(model.mpo[i], model.symm)
    sch, nidx = E.schedule_left_step(model.phys, bonds[i], bonds[i + 1], W, ch.Lidx, True)
    a = O.left_step(sch.plan, ch.Lval, ch.Lidx, t.data, t.left_paired(), nidx)
    b = REF.left_step(sch.plan, ch.Lval, ch.Lidx, t.data, t.left_paired(), nidx)
    assert np.linalg.norm(a - b) <= 1e-14 * np.linalg.norm(b)
    t = tensors[i + 1]
    W = M.MPOHandle(model.mpo[i + 1], model.symm)
    sch, nidx = E.schedule_right_step(model.phys, bonds[i + 1], bonds[i + 2], W, ch.Ridx, True)
    a = O.right_step(sch.plan, ch.Rval, ch.Ridx, t.data, t.data, nidx)
    b = REF.right_step(sch.plan, ch.Rval, ch.Ridx, t.data, t.data, nidx)
    assert np.linalg.norm(a - b) <= 1e-14 * np.linalg.norm(b)
