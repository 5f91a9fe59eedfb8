"""Spin-adapted (SU2U1) quantum chemistry on the CPU oracle.

The reference's SU2U1 path (qc_su2 terms, the bond-spin MPO, the 9j couplings of
the schedule builders, the spin-coupled two-site MPO and the spin-reduced
two-site tensor) has no golden vectors of its own, so it is pinned by exact
diagonalisation: with complete bond spaces and a mixed-canonical environment,
H_eff on the reduced two-site tensor must have exactly the spectrum of the
Hamiltonian on the spin multiplets of total (N, S) -- the FCI eigenvalues with
S^2 = S(S+1) (oracle/dense.py spin_sector_spectrum) -- plus exact zeros for the
reduced slots that no coupling path reaches; and a two-site sweep must reach
the FCI ground energy.
"""
import numpy as np
import pytest

import dense
from dmrgb200 import _capi as capi
from dmrgb200 import dmrg as G
from dmrgb200 import mps as S
from dmrgb200 import qc
from dmrgb200 import su2u1 as SU
from helpers import OracleChain, unit_mask
from sweep_backend import OracleBackend


def exact_chain(L, n_elec, two_s, seed=1):
    h, eri = qc.synthetic_integrals(L)
    model = SU.quantum_chemistry(L, n_elec, two_s, h=h, eri=eri)
    bonds = SU.allowed_sectors(L, (n_elec, two_s), 10 ** 6)
    A = S.random_mps(SU.PHYS, bonds, np.random.default_rng(seed))
    i = L // 2 - 1
    A = G.left_canonicalize(G.right_canonicalize(A), i)
    bonds = [t.left for t in A] + [A[-1].right]
    return model, bonds, A, i, h, eri


def dense_heff(ch):
    psi = S.SiteTensor(ch.p12, ch.left, ch.right)
    idx = np.nonzero(unit_mask(psi))[0]
    H = np.zeros((len(idx), len(idx)))
    for c, k in enumerate(idx):
        x = np.zeros(psi.rp.total)
        x[k] = 1.0
        H[:, c] = ch.hpsi(x)[idx]
    return H


@pytest.mark.parametrize("L,n_elec,two_s", [(4, 4, 0), (6, 6, 0), (5, 5, 1), (6, 6, 2)])
def test_heff_spectrum_equals_fci_spin_sector(L, n_elec, two_s):
    model, bonds, A, i, h, eri = exact_chain(L, n_elec, two_s)
    ch = OracleChain(model, bonds, A, i)
    H = dense_heff(ch)
    assert np.abs(H - H.T).max() < 1e-12
    ev = np.linalg.eigvalsh(0.5 * (H + H.T))
    fci = dense.spin_sector_spectrum(h, eri, n_elec, two_s)
    nz = np.sort(ev[np.abs(ev) > 1e-10])
    assert len(nz) == len(fci), (len(nz), len(fci))
    assert np.abs(nz - fci).max() < 1e-11, np.abs(nz - fci).max()
    # the remaining eigenvalues are the unreachable reduced slots (spin-1 pair on a spin-0 bond)
    assert len(ev) - len(nz) == int(np.sum(np.abs(ev) <= 1e-10))


def test_two_site_sweep_reaches_fci_ground_energy():
    L, n = 6, 6
    h, eri = qc.synthetic_integrals(L)
    model = SU.quantum_chemistry(L, n, 0, h=h, eri=eri)
    A = S.random_mps(SU.PHYS, SU.allowed_sectors(L, (n, 0), 3), np.random.default_rng(2))
    dm = G.TwoSiteDMRG(OracleBackend(), model, list(A), 100, jd_tol=1e-10, jd_maxiter=12)
    for sw in range(3):
        e = dm.sweep(sw)
    e0 = dense.spin_sector_spectrum(h, eri, n, 0)[0]
    assert abs(e - e0) < 1e-9, (e, e0)


def test_reduced_twosite_round_trip():
    """unreduce(reduce(theta)) == theta for a product-basis two-site tensor of
    physical slots (ts_reduction::reduce_right then unreduce_right: the 6j
    recoupling of the singly occupied pair is orthogonal)."""
    L, n = 6, 6
    _, bonds, A, i, _, _ = exact_chain(L, n, 0)
    p12, offs = SU.fuse_phys(SU.PHYS, SU.PHYS)
    theta = G.twosite(A[i], A[i + 1], p12, offs)
    red = SU.reduce_twosite(theta)
    back = SU.unreduce_twosite(red)
    assert np.linalg.norm(back.data - theta.data) < 1e-13 * np.linalg.norm(theta.data)
    assert abs(np.linalg.norm(red.data) - np.linalg.norm(theta.data)) < 1e-13 * np.linalg.norm(theta.data)


def test_mpo_bond_spins_follow_operator_actions():
    model = SU.quantum_chemistry(8, 8, 0)
    for W in model.mpo:
        for (b1, b2), lst in W.terms.items():
            for op, _ in lst:
                o = SU.OPS[op.name]
                assert W.right_spin[b2] == W.left_spin[b1] + o.action
                assert abs(W.left_spin[b1] - W.right_spin[b2]) <= o.K <= W.left_spin[b1] + W.right_spin[b2]
    assert model.mpo[0].left_spin == [0] and model.mpo[-1].right_spin == [0]


def test_reference_solver_core_runs_su2u1_plans():
    """The reference's own tasks.cpp (oracle/_ref) executes the SU2U1 plan as the
    oracle does: the plan carries the couplings, so the executor is symmetry-blind."""
    ref = pytest.importorskip("ref")
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    model, bonds, A, i, _, _ = exact_chain(6, 6, 0)
    ch = OracleChain(model, bonds, A, i)
    x = np.random.default_rng(5).standard_normal(int(ch.sched.plan["in_size"]))
    y_or = ch.hpsi(x)
    y_ref = ref.hpsi(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, x)
    assert np.linalg.norm(y_or - y_ref) <= 1e-14 * np.linalg.norm(y_ref)
    assert ch.sched.plan["kind"] == capi.PLAN_HPSI


def test_two_fci_references_agree():
    """The determinant FCI (E_pq algebra, S+ null space) used above against the dense
    spin-orbital Hamiltonian of the TwoU1 model with an explicit S^2 (independent
    constructions of the same spectrum)."""
    h, eri = qc.synthetic_integrals(4)
    for n, s in ((4, 0), (3, 1)):
        a = dense.spin_sector_spectrum(h, eri, n, s)
        b = dense.spin_sector_spectrum_jw(h, eri, n, s)
        assert len(a) == len(b) and np.abs(a - b).max() < 1e-12
