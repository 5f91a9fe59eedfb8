"""Adjoint of H·psi on the CPU oracle and the builder's term provenance.

The product is y = sum_k alpha_k H_k x over the plan terms; its adjoint gives
gx = H^T w and galpha_k = <w|H_k x>.  Checked here without a GPU: exact
identities of the transpose, central finite differences in alpha and in the MPO
term scales (through dmrgb200_schedule_term_sources), and the physical meaning of
the coefficient gradient: d<psi|H_eff|psi>/dt and d/dU equal the hopping
expectation and the double occupancy of the embedded state (1-/2-RDM elements)
from the dense Hamiltonian."""
import dataclasses

import numpy as np
import pytest

from dmrgb200 import engine as E
from dmrgb200 import models as M

import oracle as O
import dense as D
from helpers import (OracleChain, hubbard_center_terms, hubbard_derivative_ops, make_chain, perturbed_mpo,
                     random_psi)


def _chain(name="hubbard", L=6, Mmax=8, i=2, seed=11, merge=True):
    model, bonds, tensors, rng = make_chain(name, L, Mmax, seed=seed)
    return OracleChain(model, bonds, tensors, i, merge=merge), rng


@pytest.mark.parametrize("name", ["hubbard", "heisenberg", "bose"])
def test_adjoint_identities(name):
    ch, rng = _chain(name, L=6 if name != "heisenberg" else 8)
    p = ch.sched.plan
    w = random_psi(ch.p12, ch.left, ch.right, rng).data
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    gx, ga = O.hpsi_adjoint(p, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, w, x)
    hx, hw = ch.hpsi(x), ch.hpsi(w)
    ref = w @ hx
    scale = np.linalg.norm(w) * np.linalg.norm(hx)
    # transpose: <H^T w, x> = <w, H x>
    assert abs(gx @ x - ref) <= 1e-12 * scale
    # linearity in the terms: sum_k alpha_k <w|H_k x> = <w|H x>
    assert abs(p["term_alpha"] @ ga - ref) <= 1e-12 * scale
    # Hermitian effective Hamiltonian: H^T w = H w
    assert np.linalg.norm(gx - hw) <= 1e-12 * np.linalg.norm(hw)


def test_galpha_central_differences():
    ch, rng = _chain()
    p = ch.sched.plan
    w = random_psi(ch.p12, ch.left, ch.right, rng).data
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    _, ga = O.hpsi_adjoint(p, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, w, x)
    h = 1e-6
    for k in rng.choice(len(p["term_alpha"]), size=12, replace=False):
        f = []
        for sgn in (1, -1):
            q = dict(p)
            q["term_alpha"] = p["term_alpha"].copy()
            q["term_alpha"][k] += sgn * h
            f.append(w @ O.hpsi(q, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, x))
        fd = (f[0] - f[1]) / (2 * h)
        assert abs(fd - ga[k]) <= 1e-7 * max(1.0, abs(ga[k])), (k, fd, ga[k])


@pytest.mark.parametrize("merge", [True, False])
def test_mpo_term_scale_gradient(merge):
    """d<w|H x>/d(term scale) from galpha and the schedule's term provenance
    against central differences of rebuilt schedules."""
    ch, rng = _chain(merge=merge)
    w = random_psi(ch.p12, ch.left, ch.right, rng).data
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    _, ga = O.hpsi_adjoint(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, w, x)
    g = ch.sched.mpo_term_grad(ga, ch.W12.n_terms)
    h = 1e-5
    for idx in range(ch.W12.n_terms):
        f = []
        for sgn in (1, -1):
            Wp = M.MPOHandle(perturbed_mpo(ch.W12mpo, ch.W12.term_keys[idx], sgn * h), ch.model.symm)
            s = E.schedule_hpsi(ch.p12, ch.left, ch.right, Wp, ch.Lidx, ch.Ridx)
            f.append(w @ O.hpsi(s.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, x))
        fd = (f[0] - f[1]) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-7 * max(1.0, abs(g[idx])), (idx, fd, g[idx])


def test_coefficient_gradient_is_local_rdm():
    """d<psi|H_eff|psi>/dt (centre bond) and d/dU (centre sites) from the adjoint
    equal <P psi| dH/dc |P psi> of the dense Hamiltonian: the hopping 1-RDM element
    and the double occupancy (2-RDM diagonal)."""
    L, i = 6, 2
    ch, rng = _chain(L=L, i=i, merge=False)
    psi = random_psi(ch.p12, ch.left, ch.right, rng).data
    _, ga = O.hpsi_adjoint(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, psi, psi)
    g = ch.sched.mpo_term_grad(ga, ch.W12.n_terms)
    sel = hubbard_center_terms(ch.W12, ch.W12mpo)
    coeff = {"t": 1.0, "U1": 4.0, "U2": 4.0}    # fermi_hubbard defaults
    P = D.embedding(ch.tensors[:i], ch.tensors[i + 2:], ch.model.phys, ch.model.phys, ch.left, ch.right, ch.p12)
    v = P @ psi
    for name, terms in hubbard_derivative_ops(ch.model, i).items():
        assert sel[name], name
        grad = sum(g[j] * ch.W12.term_scale[j] / coeff[name] for j in sel[name])
        Op = D.sparse_hamiltonian(dataclasses.replace(ch.model, dense_terms=terms), L)
        expect = v @ (Op @ v)
        assert abs(grad - expect) <= 1e-11 * max(1.0, abs(expect)), (name, grad, expect)
