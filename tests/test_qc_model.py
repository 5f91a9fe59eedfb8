"""Quantum-chemistry Hamiltonian (TwoU1, spatial orbitals): the bipartite-graph
MPO reproduces the dense Hamiltonian built from the integrals with explicit
Jordan-Wigner strings, and the schedule + oracle H·psi reproduce P^T H P of a
two-site problem (FP64, 1e-12)."""
import numpy as np
import pytest

import dense as D
from dmrgb200 import qc
from helpers import OracleChain, make_chain, random_psi


@pytest.mark.parametrize("L", [3, 4, 5])
def test_qc_mpo_reproduces_dense_hamiltonian(L):
    m = qc.quantum_chemistry(L, L // 2, L - L // 2)
    H = D.dense_hamiltonian(m, L)
    assert np.abs(H - H.T).max() <= 1e-13 * np.abs(H).max()
    Hm = D.mpo_dense(m, L)
    assert np.abs(Hm - H).max() <= 1e-12 * np.abs(H).max()


def test_qc_mpo_bond_dimension():
    """The bipartite-graph construction stays at the 2 L^2 + 4 L + 2 channels of the
    complementary-operator QC MPO in the middle of the chain (22 at the ends)."""
    h, eri = qc.synthetic_integrals(8)
    mpo = qc.build_mpo(qc.qc_terms(h, eri), 8, qc.local_ops(), qc.PHYS)
    dims = [w.col_dim for w in mpo]
    assert dims[0] == 22 and dims[-1] == 1 and max(dims) <= 2 * 8 * 8 + 4 * 8 + 2


@pytest.mark.parametrize("i", [0, 2])
def test_qc_heff_matches_dense(i):
    L = 5
    model, bonds, tensors, rng = make_chain("qc", L, 16, seed=12)
    ch = OracleChain(model, bonds, tensors, i)
    psi = random_psi(ch.p12, ch.left, ch.right, rng)
    y = ch.hpsi(psi.data)
    H = D.sparse_hamiltonian(model, L)
    P = D.embedding(tensors[:i], tensors[i + 2:], model.phys, model.phys, ch.left, ch.right, ch.p12)
    yd = P.T @ (H @ (P @ psi.data))
    assert np.linalg.norm(y - yd) <= 1e-12 * np.linalg.norm(yd)


# integrals whose every operator sits at or left of the centre pair (sites 1, 2 of
# L = 5): their coefficient is placed in the centre MPO tensors, so the local
# adjoint gives the whole derivative, a 1- or 2-RDM element of the embedded state
LOCAL_INTEGRALS = [("h", (1, 2)), ("h", (1, 1)), ("h", (2, 2)), ("h", (0, 2)),
                   ("eri", (1, 1, 2, 2)), ("eri", (1, 2, 1, 2)), ("eri", (0, 1, 2, 2)), ("eri", (2, 2, 2, 2))]


@pytest.mark.parametrize("which,index", LOCAL_INTEGRALS)
def test_qc_integral_derivative_is_local_rdm(which, index):
    import dataclasses

    import oracle as O
    from helpers import qc_integral_derivative
    L, i = 5, 1
    model, bonds, tensors, rng = make_chain("qc", L, 16, seed=12)
    ch = OracleChain(model, bonds, tensors, i)
    psi = random_psi(ch.p12, ch.left, ch.right, rng).data
    _, ga = O.hpsi_adjoint(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, psi, psi)
    grad, terms = qc_integral_derivative(model, L, i, ch, ga, which, index)
    P = D.embedding(tensors[:i], tensors[i + 2:], model.phys, model.phys, ch.left, ch.right, ch.p12)
    v = P @ psi
    Op = D.sparse_hamiltonian(dataclasses.replace(model, dense_terms=terms), L)
    expect = v @ (Op @ v)
    assert abs(grad - expect) <= 1e-11 * max(1.0, abs(expect)), (which, index, grad, expect)


@pytest.mark.parametrize("which,index", [("h", (0, 2)), ("eri", (0, 1, 2, 3)), ("eri", (1, 1, 2, 2))])
def test_operator_model_mpo_reproduces_dense_operator(which, index):
    """The MPO of dH/d(integral) (the observable of the RDM element) matches the
    dense operator built from the same term list."""
    import dataclasses
    L = 4
    model = qc.quantum_chemistry(L, 2, 2)
    terms = qc.integral_operator_terms(which, index)
    om = qc.operator_model(model, terms)
    dense = D.dense_hamiltonian(dataclasses.replace(model, dense_terms=terms), L)
    assert np.abs(D.mpo_dense(om, L) - dense).max() <= 1e-12 * max(1.0, np.abs(dense).max())


@pytest.mark.parametrize("which,index", [("h", (0, 2)), ("eri", (0, 1, 2, 2))])
def test_integral_derivative_equals_operator_expectation(which, index):
    """The local adjoint derivative equals <psi|H_eff(dH/d(integral))|psi>, the RDM
    element computed through the observable's own MPO, boundaries and schedule
    (the check used at L = 16 on the device)."""
    import oracle as O
    from helpers import qc_integral_derivative
    L, i = 5, 1
    model, bonds, tensors, rng = make_chain("qc", L, 16, seed=12)
    ch = OracleChain(model, bonds, tensors, i)
    psi = random_psi(ch.p12, ch.left, ch.right, rng).data
    _, ga = O.hpsi_adjoint(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, psi, psi)
    grad, terms = qc_integral_derivative(model, L, i, ch, ga, which, index)
    oc = OracleChain(qc.operator_model(model, terms), bonds, tensors, i)
    expect = float(psi @ oc.hpsi(psi))
    assert abs(grad - expect) <= 1e-11 * max(1.0, abs(expect)), (grad, expect)


def test_integral_file_round_trip(tmp_path):
    """The reference's integral text format (unique entries, 1-based, 0 for absent
    indices) and its binary buffer both read back the synthetic integrals exactly."""
    L = 5
    h, eri = qc.synthetic_integrals(L)
    path = tmp_path / "FCIDUMP"
    n = qc.write_integrals(path, h, eri, core=1.25)
    P = L * (L + 1) // 2
    assert n == P * (P + 1) // 2 + P + 1
    lines = path.read_text().splitlines()
    assert len(lines) == 4 + n and lines[-1].split()[1:] == ["0", "0", "0", "0"]
    h2, eri2, core = qc.read_integrals(path, L)
    assert np.array_equal(h2, h) and np.array_equal(eri2, eri) and core == 1.25
    h3, eri3, core3 = qc.parse_integrals_buffer(qc.integrals_buffer(h, eri, core=1.25), L)
    assert np.array_equal(h3, h) and np.array_equal(eri3, eri) and core3 == 1.25


def test_integral_file_orbital_order(tmp_path):
    """orbital_order (1-based, the orbital placed at each site) permutes the integrals."""
    L = 4
    h, eri = qc.synthetic_integrals(L)
    path = tmp_path / "FCIDUMP"
    qc.write_integrals(path, h, eri)
    order = [3, 1, 4, 2]
    h2, eri2, _ = qc.read_integrals(path, L, order=order)
    o = np.array(order) - 1
    assert np.array_equal(h2, h[np.ix_(o, o)])
    assert np.array_equal(eri2, eri[np.ix_(o, o, o, o)])


def test_integral_file_cutoff_and_errors(tmp_path):
    L = 3
    h, eri = qc.synthetic_integrals(L)
    path = tmp_path / "FCIDUMP"
    qc.write_integrals(path, h, eri)
    h2, eri2, _ = qc.read_integrals(path, L, cutoff=0.05)
    keep = np.abs(eri) > 0.05
    assert np.array_equal(eri2[keep], eri[keep]) and not np.any(eri2[~keep])
    assert np.array_equal(h2[np.abs(h) > 0.05], h[np.abs(h) > 0.05])
    bad = tmp_path / "bad"
    bad.write_text("a\nb\nc\nd\n1.0 1 1 0\n")
    with pytest.raises(ValueError):
        qc.read_integrals(bad, L)
    with pytest.raises(ValueError):
        qc.parse_integrals_buffer(b"\0" * 23, L)
