"""Jacobi-Davidson on the device (dmrgb200_solve) against the oracle's numpy
restatement of the reference's solver, and against dense eigenvalues."""
import numpy as np
import pytest

import dense as D
import jd as JD
from dmrgb200 import _capi as capi
from dmrgb200 import engine as E
from dmrgb200 import mps as S
from helpers import OracleChain, make_chain, random_psi, unit_mask

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


MODES = [capi.SOLVER_GRAPH, capi.SOLVER_STEPWISE]


def _setup(name, L, i, seed, mode=capi.SOLVER_GRAPH, **kw):
    model, bonds, tensors, rng = make_chain(name, L, kw.get("Mmax", 0), seed=seed, synthetic_m=kw.get("m"))
    ch = OracleChain(model, bonds, tensors, i)
    ctx = E.Context(0)
    Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
    plan = E.DevicePlan(ctx, ch.sched.plan, left_addr=ch.Lidx.cohort_addresses(Lb.data_ptr()),
                        other_addr=ch.Ridx.cohort_addresses(Rb.data_ptr()))
    plan.set_solver(mode)
    x0 = random_psi(ch.p12, ch.left, ch.right, rng).data
    return ch, plan, (ctx, Lb, Rb), x0, rng


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("max_iter", [1, 2, 5, 8])
def test_solve_matches_oracle_iteration_by_iteration(max_iter, mode):
    ch, plan, keep, x0, rng = _setup("hubbard", 12, 5, seed=31, mode=mode, m=48)
    theta_ref, u_ref, it_ref, conv_ref, r_ref = JD.jcd(ch.hpsi, x0, tol=1e-10, max_iter=max_iter)
    xd = E.to_device(x0)
    xo = torch.zeros_like(xd)
    theta, st = plan.solve(xd.data_ptr(), xo.data_ptr(), xd.numel(), tol=1e-10, max_iter=max_iter)
    assert st.iterations == it_ref
    assert abs(theta - theta_ref) <= 1e-11 * abs(theta_ref)
    u = xo.cpu().numpy()
    s = np.sign(u @ u_ref)
    assert np.linalg.norm(s * u - u_ref) <= 1e-9 * np.linalg.norm(u_ref)
    assert abs(st.residual - r_ref) <= 1e-8 * max(r_ref, 1e-12) + 1e-14


@pytest.mark.parametrize("mode", MODES)
def test_solve_reaches_dense_lowest_eigenvalue(mode):
    ch, plan, keep, x0, rng = _setup("heisenberg", 6, 2, seed=2, mode=mode, Mmax=4)
    m = unit_mask(S.SiteTensor(ch.p12, ch.left, ch.right))
    P = D.embedding(ch.tensors[:2], ch.tensors[4:], ch.model.phys, ch.model.phys, ch.left, ch.right, ch.p12)
    H = D.dense_hamiltonian(ch.model, 6)
    Heff = (P.T @ H @ P)[np.ix_(m, m)]
    lam = np.linalg.eigvalsh(Heff)[0]
    xd = E.to_device(x0)
    xo = torch.zeros_like(xd)
    theta, st = plan.solve(xd.data_ptr(), xo.data_ptr(), xd.numel(), tol=1e-12, max_iter=min(32, int(m.sum())))
    assert theta >= lam - 1e-10 * abs(lam)
    assert abs(theta - lam) <= 1e-9 * abs(lam)


@pytest.mark.parametrize("mode", MODES)
def test_solve_with_orthogonal_vectors(mode):
    ch, plan, keep, x0, rng = _setup("hubbard", 10, 4, seed=8, mode=mode, m=32)
    o1 = random_psi(ch.p12, ch.left, ch.right, rng).data
    o2 = random_psi(ch.p12, ch.left, ch.right, rng).data
    theta_ref, u_ref, it_ref, _, _ = JD.jcd(ch.hpsi, x0, ortho=[o1, o2], tol=1e-10, max_iter=6)
    xd, od1, od2 = E.to_device(x0), E.to_device(o1), E.to_device(o2)
    xo = torch.zeros_like(xd)
    theta, st = plan.solve(xd.data_ptr(), xo.data_ptr(), xd.numel(), ortho_ptrs=[od1.data_ptr(), od2.data_ptr()],
                           tol=1e-10, max_iter=6)
    assert abs(theta - theta_ref) <= 1e-11 * abs(theta_ref)
    u = xo.cpu().numpy()
    assert abs(u @ o1) <= 1e-10 * np.linalg.norm(u) * np.linalg.norm(o1)


def test_graph_solver_reused_and_reproducible():
    """The cached solver graph serves repeated solves with new start vectors;
    identical inputs give bitwise identical results, and both modes agree."""
    ch, plan, keep, x0, rng = _setup("hubbard", 12, 5, seed=33, m=48)
    x1 = random_psi(ch.p12, ch.left, ch.right, rng).data
    outs = []
    for x in (x0, x1, x0):
        xd = E.to_device(x)
        xo = torch.zeros_like(xd)
        theta, st = plan.solve(xd.data_ptr(), xo.data_ptr(), xd.numel(), tol=1e-10, max_iter=8)
        assert st.solve_ms > 0
        outs.append((theta, xo.cpu().numpy(), st.iterations))
    assert outs[0][0] == outs[2][0] and np.array_equal(outs[0][1], outs[2][1])
    theta_ref, u_ref, it_ref, _, _ = JD.jcd(ch.hpsi, x1, tol=1e-10, max_iter=8)
    assert outs[1][2] == it_ref and abs(outs[1][0] - theta_ref) <= 1e-11 * abs(theta_ref)
    plan.set_solver(capi.SOLVER_STEPWISE)
    xd = E.to_device(x0)
    xo = torch.zeros_like(xd)
    theta, st = plan.solve(xd.data_ptr(), xo.data_ptr(), xd.numel(), tol=1e-10, max_iter=8)
    assert abs(theta - outs[0][0]) <= 1e-12 * abs(theta) and st.iterations == outs[0][2]
