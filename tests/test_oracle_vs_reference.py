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


FLAT_KEYS = ("g_t", "g_c", "in_rows", "in_cols", "in_off", "out_rows", "out_cols", "out_off", "t_lb", "t_col", "t_ci",
             "t_trans", "t_nb", "t_brows", "t_bcols", "c_lb", "c_rb", "c_ls", "c_rs", "c_ci", "c_trans", "c_nsrows",
             "c_stripe", "c_unit", "u_offset", "u_ms", "u_line", "l_b1", "l_term", "term_alpha", "term_t",
             "term_col")


@pytest.mark.parametrize("name,L,m", [("hubbard", 10, 40), ("qc", 8, 32), ("su2u1", 8, 48)])
def test_reference_schedule_flattens_to_the_same_plan(name, L, m):
    """The drop-in seam end to end on the host: a flat plan is replayed into the
    reference's own ScheduleNew / MPSBlock / Cohort objects (ref_adapter.cpp), the
    reference-side flattener (ref_flatten.cpp) turns that ScheduleNew back into a
    dmrgb200_plan_desc, and every array comes back identical -- so a caller that
    builds its schedules with the reference's code hands libdmrgb200 exactly the
    plan the library's own builder produces (the H·psi parity of that plan is
    covered on the GPU)."""
    if name == "su2u1":
        from dmrgb200 import mps as S
        from dmrgb200 import su2u1 as SU
        model = SU.quantum_chemistry(L, L, 0)
        bonds = SU.synthetic_bonds(L, (L, 0), m)
        tensors = S.random_mps(SU.PHYS, bonds, np.random.default_rng(5))
    else:
        model, bonds, tensors, _ = make_chain(name, L, 0, seed=5, synthetic_m=m)
    ch = OracleChain(model, bonds, tensors, L // 2 - 1)
    h = REF.Hpsi(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx)
    flat = h.flatten()
    for k in FLAT_KEYS:
        assert np.array_equal(np.asarray(flat[k]), np.asarray(ch.sched.plan[k])), k
    assert flat["in_size"] == ch.sched.plan["in_size"] and flat["out_size"] == ch.sched.plan["out_size"]
    # the reference's CPU execution accumulates output blocks under mutexes in thread order,
    # so two runs agree to rounding, not bitwise
    x = np.random.default_rng(1).standard_normal(int(flat["in_size"]))
    a, b = h.run(x), REF.hpsi(flat, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, x)
    assert np.linalg.norm(a - b) <= 1e-14 * np.linalg.norm(b)
