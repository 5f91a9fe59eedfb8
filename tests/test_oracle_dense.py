"""The oracle (CPU restatement of the reference's schedule execution) driven by
the library's schedule builder reproduces the dense effective Hamiltonian
P^T H P of small chains to machine precision (FP64, relative 1e-12)."""
import numpy as np
import pytest

import dense as D
from helpers import OracleChain, make_chain, random_psi

TOL = 1e-12

CASES = [("heisenberg", 6, 4), ("hubbard", 4, 4), ("bose", 5, 3)]


@pytest.mark.parametrize("name,L,Mmax", CASES)
@pytest.mark.parametrize("symmetric", [True, False])
def test_hpsi_matches_dense_heff(name, L, Mmax, symmetric):
    model, bonds, tensors, rng = make_chain(name, L, Mmax, seed=11)
    H = D.dense_hamiltonian(model, L)
    for i in range(L - 1):
        ch = OracleChain(model, bonds, tensors, i, symmetric)
        psi = random_psi(ch.p12, ch.left, ch.right, rng)
        y = ch.hpsi(psi.data)
        P = D.embedding(tensors[:i], tensors[i + 2:], model.phys, model.phys, ch.left, ch.right, ch.p12)
        yd = P.T @ (H @ (P @ psi.data))
        assert np.linalg.norm(y - yd) <= TOL * np.linalg.norm(yd), (name, i)


@pytest.mark.parametrize("name,L,Mmax", CASES)
def test_mpo_reproduces_dense_hamiltonian(name, L, Mmax):
    """Contracting the site MPOs over the full basis gives the directly built H."""
    model, bonds, tensors, rng = make_chain(name, L, Mmax)
    H = D.dense_hamiltonian(model, L)
    Hm = D.mpo_dense(model, L)
    assert np.allclose(Hm, H, atol=1e-12)


def test_heff_is_symmetric():
    """<x|H y> = <H x|y> (the reference's Hermiticity of the site problem)."""
    model, bonds, tensors, rng = make_chain("hubbard", 6, 6, seed=3)
    ch = OracleChain(model, bonds, tensors, 2)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    y = random_psi(ch.p12, ch.left, ch.right, rng).data
    assert abs(x @ ch.hpsi(y) - ch.hpsi(x) @ y) <= 1e-12 * np.linalg.norm(x) * np.linalg.norm(ch.hpsi(y))


def test_symmetric_and_full_boundaries_agree():
    model, bonds, tensors, rng = make_chain("heisenberg", 8, 6, seed=5)
    a = OracleChain(model, bonds, tensors, 3, symmetric=True)
    b = OracleChain(model, bonds, tensors, 3, symmetric=False)
    x = random_psi(a.p12, a.left, a.right, rng).data
    ya, yb = a.hpsi(x), b.hpsi(x)
    assert np.linalg.norm(ya - yb) <= 1e-13 * np.linalg.norm(ya)


def test_bose_hubbard_model_matches_reference_known_answer():
    """The reference's coded Bose-Hubbard regression test
    (regression/applications/dmrg/test_coded_bh_ts.py:16-53) quotes
    E = -6.881090360639349 (tolerance 1e-3) for L=10, Nmax=2, t=1, U=8, N=5.
    Exact diagonalisation of the model as built here reproduces it."""
    from dmrgb200 import models as M
    e = D.ground_energy(M.bose_hubbard(10, t=1.0, U=8.0, Nmax=2, N=5), 10)
    assert abs(e - (-6.881090360639349)) <= 1e-9
