"""Jacobi-Davidson on the device (dmrgb200_solve) against the oracle's numpy
restatement of the reference's solver, and against dense eigenvalues."""
import numpy as np
import pytest

import dense as D
import jd as JD
from dmrgb200 import engine as E
from dmrgb200 import mps as S
from helpers import OracleChain, make_chain, random_psi, unit_mask

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _setup(name, L, i, seed, **kw):
    model, bonds, tensors, rng = make_chain(name, L, kw.get("Mmax", 0), seed=seed, synthetic_m=kw.get("m"))
    ch = OracleChain(model, bonds, tensors, i)
    ctx = E.Context(0)
    Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
    plan = E.DevicePlan(ctx, ch.sched.plan, left_addr=ch.Lidx.cohort_addresses(Lb.data_ptr()),
                        other_addr=ch.Ridx.cohort_addresses(Rb.data_ptr()))
    x0 = random_psi(ch.p12, ch.left, ch.right, rng).data
    return ch, plan, (ctx, Lb, Rb), x0, rng


@pytest.mark.parametrize("max_iter", [1, 2, 5, 8])
def test_solve_matches_oracle_iteration_by_iteration(max_iter):
    ch, plan, keep, x0, rng = _setup("hubbard", 12, 5, seed=31, m=48)
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


def test_solve_reaches_dense_lowest_eigenvalue():
    ch, plan, keep, x0, rng = _setup("heisenberg", 6, 2, seed=2, Mmax=4)
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


def test_solve_with_orthogonal_vectors():
    ch, plan, keep, x0, rng = _setup("hubbard", 10, 4, seed=8, m=32)
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
