"""Quantum-chemistry Hamiltonian on the device path: H·psi and boundary steps
against the CPU oracle (FP64, 1e-12), two-site DMRG sweeps against exact
diagonalisation (1e-9), and integral derivatives through the device adjoint
against the dense 1-/2-RDM elements of the embedded state."""
import dataclasses

import numpy as np
import pytest

import dense as D
import oracle as O
from dmrgb200 import dmrg as G
from dmrgb200 import engine as E
from dmrgb200 import mps as S
from dmrgb200 import qc
from helpers import OracleChain, make_chain, qc_integral_derivative, random_psi

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return E.Context(0)


def _plan(ctx, ch):
    Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
    plan = E.DevicePlan(ctx, ch.sched.plan, left_addr=ch.Lidx.cohort_addresses(Lb.data_ptr()),
                        other_addr=ch.Ridx.cohort_addresses(Rb.data_ptr()))
    return plan, (Lb, Rb)


@pytest.mark.parametrize("L,m,i", [(8, 64, 3), (10, 48, 2)])
def test_qc_hpsi_matches_oracle(ctx, L, m, i):
    model, bonds, tensors, rng = make_chain("qc", L, 0, seed=5, synthetic_m=m)
    ch = OracleChain(model, bonds, tensors, i)
    plan, keep = _plan(ctx, ch)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    xd = E.to_device(x)
    yd = torch.zeros_like(xd)
    plan.hpsi(xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    ref = ch.hpsi(x)
    assert np.linalg.norm(yd.cpu().numpy() - ref) <= 1e-12 * np.linalg.norm(ref)


def test_qc_sweeps_reach_exact_ground_state(ctx):
    L = 6
    model = qc.quantum_chemistry(L, 3, 3)
    rng = np.random.default_rng(2)
    bonds = S.allowed_sectors(model.phys, L, model.total_charge, 5)
    A = S.random_mps(model.phys, bonds, rng)
    opt = G.TwoSiteDMRG(G.DeviceBackend(ctx), model, A, 64, cutoff=1e-16, jd_tol=1e-10, jd_maxiter=16)
    e = None
    for s in range(4):
        e = opt.sweep(s)
    assert abs(e - D.ground_energy(model, L)) <= 1e-9


@pytest.mark.parametrize("which,index", [("h", (1, 2)), ("h", (0, 2)), ("eri", (1, 1, 2, 2)), ("eri", (0, 1, 2, 2))])
def test_qc_integral_derivative_on_device(ctx, which, index):
    L, i = 5, 1
    model, bonds, tensors, rng = make_chain("qc", L, 16, seed=12)
    ch = OracleChain(model, bonds, tensors, i)
    plan, keep = _plan(ctx, ch)
    psi = random_psi(ch.p12, ch.left, ch.right, rng).data
    xd = E.to_device(psi)
    ga = torch.empty(len(ch.sched.plan["term_alpha"]), dtype=torch.float64, device="cuda")
    plan.adjoint(xd.data_ptr(), xd.data_ptr(), 0, ga.data_ptr())
    torch.cuda.synchronize()
    ga = ga.cpu().numpy()
    _, ga_o = O.hpsi_adjoint(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, psi, psi)
    assert np.linalg.norm(ga - ga_o) <= 1e-12 * np.linalg.norm(ga_o)
    grad, terms = qc_integral_derivative(model, L, i, ch, ga, which, index)
    P = D.embedding(tensors[:i], tensors[i + 2:], model.phys, model.phys, ch.left, ch.right, ch.p12)
    v = P @ psi
    Op = D.sparse_hamiltonian(dataclasses.replace(model, dense_terms=terms), L)
    expect = v @ (Op @ v)
    assert abs(grad - expect) <= 1e-11 * max(1.0, abs(expect))
