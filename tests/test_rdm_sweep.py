"""Integral derivatives (1-/2-RDM elements) of a whole MPS by moving the two-site
centre over every site pair (dmrgb200.rdm) on the CPU oracle, against the dense
expectation value <psi|dH/dc|psi> of the normalised state -- including integrals
whose coefficients sit far from any one centre pair."""
import dataclasses

import numpy as np

import dense as D
from dmrgb200 import mps as S
from dmrgb200 import qc
from dmrgb200 import rdm
from sweep_backend import OracleBackend

INTEGRALS = [("h", (0, 1)), ("h", (3, 4)), ("h", (0, 4)), ("h", (2, 2)), ("eri", (0, 0, 4, 4)),
             ("eri", (0, 1, 3, 4)), ("eri", (1, 2, 2, 3)), ("eri", (0, 3, 1, 4))]


def dense_derivatives(model, tensors, L):
    v = D.mps_dense([t.dense() for t in tensors])
    v = v / np.linalg.norm(v)
    out = {}
    for key in INTEGRALS:
        Op = D.sparse_hamiltonian(dataclasses.replace(model, dense_terms=qc.integral_operator_terms(*key)), L)
        out[key] = float(v @ (Op @ v))
    return out


def test_integral_derivatives_over_the_chain_match_dense_rdm_elements():
    L = 5
    model = qc.quantum_chemistry(L, 2, 2)
    tensors = S.random_mps(model.phys, S.allowed_sectors(model.phys, L, model.total_charge, 16),
                           np.random.default_rng(7))
    got = rdm.integral_derivatives(OracleBackend(), model, tensors, INTEGRALS)
    want = dense_derivatives(model, tensors, L)
    for key in INTEGRALS:
        assert abs(got[key] - want[key]) <= 1e-11 * max(1.0, abs(want[key])), (key, got[key], want[key])


def test_su2u1_integral_derivatives_match_unit_integral_models():
    """SU2U1: the derivative of E for the normalised MPS equals <psi|H(unit integral)|psi>,
    the energy of the model whose only integral is the raised one (H is linear in the
    integrals), evaluated through that model's own MPO and boundaries."""
    from dmrgb200 import dmrg as G
    from dmrgb200 import su2u1 as SU
    from helpers import OracleChain
    L, n = 6, 6
    h, eri = qc.synthetic_integrals(L)
    model = SU.quantum_chemistry(L, n, 0, h=h, eri=eri)
    A = S.random_mps(SU.PHYS, SU.allowed_sectors(L, (n, 0), 12), np.random.default_rng(1))
    ints = [("h", (2, 3)), ("h", (0, 3)), ("h", (0, 5)), ("eri", (2, 3, 2, 3)), ("eri", (0, 1, 4, 5)),
            ("eri", (1, 2, 3, 3))]
    got = rdm.integral_derivatives(OracleBackend(), model, A, ints)
    C = G.right_canonicalize(list(A), 0.0)
    bonds = [t.left for t in C] + [C[-1].right]
    for key in ints:
        h1, e1 = qc.raise_integral(np.zeros_like(h), np.zeros_like(eri), key[0], key[1], 1.0)
        ch = OracleChain(rdm.with_integrals(model, h1, e1), bonds, C, 0)
        p12, offs = SU.fuse_phys(SU.PHYS, SU.PHYS)
        theta = SU.reduce_twosite(G.twosite(C[0], C[1], p12, offs), SU.PHYS, SU.PHYS, offs).data
        want = float(theta @ ch.hpsi(theta)) / float(theta @ theta)
        assert abs(got[key] - want) <= 1e-11 * max(1.0, abs(want)), (key, got[key], want)
