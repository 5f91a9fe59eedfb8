"""State prediction (density-matrix perturbation) of the two-site split on the CPU.

The perturbation terms alpha sum S S^T / alpha sum S^T S are pinned to the
reference's own Cohort::lbtm / rbtm (oracle/_ref, tasks.cpp:346-380) on step plans
of the two-site tensor viewed as one site (prediction.hpp:152-212); the split built
on them (dmrg.predict_split) reduces to the SVD split at alpha = 0, and perturbed
sweeps reach exact diagonalisation."""
import numpy as np
import pytest

import dense
import oracle as O
from dmrgb200 import dmrg as G
from dmrgb200 import engine as E
from dmrgb200 import models as M
from dmrgb200 import mps as S
from dmrgb200 import qc
from dmrgb200 import su2u1 as SU
from helpers import OracleChain, make_chain, random_psi
from sweep_backend import OracleBackend


def site_pair(name, L=8, m=12, seed=4):
    if name == "su2u1":
        h, eri = qc.synthetic_integrals(L)
        model = SU.quantum_chemistry(L, L, 0, h=h, eri=eri)
        bonds = SU.synthetic_bonds(L, (L, 0), m)
        rng = np.random.default_rng(seed)
        tensors = S.random_mps(SU.PHYS, bonds, rng)
    else:
        model, bonds, tensors, rng = make_chain(name, L, m, seed=seed)
    i = L // 2 - 1
    ch = OracleChain(model, bonds, tensors, i)
    psi = random_psi(ch.p12, ch.left, ch.right, rng)
    return model, ch, psi, i


def step_plan(model, ch, t, i, left):
    if left:
        W = M.MPOHandle(model.mpo[i], model.symm)
        sch, _ = E.schedule_left_step(model.phys, t.left, t.right, W, ch.Lidx, False)
        return sch.plan, ch.Lval, ch.Lidx, t.data, t.left_paired()
    W = M.MPOHandle(model.mpo[i + 1], model.symm)
    sch, _ = E.schedule_right_step(model.phys, t.left, t.right, W, ch.Ridx, False)
    return sch.plan, ch.Rval, ch.Ridx, t.data, t.data


@pytest.mark.parametrize("name", ["heisenberg", "hubbard", "su2u1"])
@pytest.mark.parametrize("left", [True, False])
def test_perturbation_terms_match_reference_lbtm_rbtm(name, left):
    ref = pytest.importorskip("ref")
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    model, ch, psi, i = site_pair(name)
    p12, offs = M.fuse_phys(model.phys, model.phys)
    t, _ = G.theta_site(psi, model.phys, model.phys, offs, left)
    plan, B, Bidx, ket, bra = step_plan(model, ch, t, i, left)
    ours = O.alpha_dm(plan, B, Bidx, ket, bra, 0.3, with_theta=False)
    theirs = ref.alpha_dm(plan, B, Bidx, ket, 0.3)
    num = sum(float(np.linalg.norm(a - b) ** 2) for a, b in zip(ours, theirs))
    den = sum(float(np.linalg.norm(b) ** 2) for b in theirs)
    assert den > 0 and np.sqrt(num / den) <= 1e-13, np.sqrt(num / den)


@pytest.mark.parametrize("left", [True, False])
def test_theta_term_is_the_plain_density_matrix(left):
    """alpha = 0: dm of every middle charge is Theta Theta^T (Theta^T Theta), Theta the
    matrix the SVD split factorises (the bra blocks of theta_site are Theta)."""
    model, ch, psi, i = site_pair("hubbard")
    p12, offs = M.fuse_phys(model.phys, model.phys)
    t, mids = G.theta_site(psi, model.phys, model.phys, offs, left)
    plan, B, Bidx, ket, bra = step_plan(model, ch, t, i, left)
    dm = O.alpha_dm(plan, B, Bidx, ket, bra, 0.0)
    for b, mc in enumerate(sorted(mids)):
        rows, cols, nr, nc, fills = mids[mc]
        Th = np.zeros((nr, nc))
        for (ro, co, ml, mr, lb, c0) in fills:
            Th[ro:ro + ml, co:co + mr] = S.block_view(psi.data, psi.rp, lb)[:, c0:c0 + mr]
        want = Th @ Th.T if left else Th.T @ Th
        assert np.abs(dm[b] - want).max() <= 1e-13 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("left", [True, False])
def test_predict_split_at_alpha_zero_is_the_svd_split(left):
    model, ch, psi, i = site_pair("heisenberg", L=8, m=16)
    p12, offs = M.fuse_phys(model.phys, model.phys)
    t, _ = G.theta_site(psi, model.phys, model.phys, offs, left)
    plan, B, Bidx, ket, bra = step_plan(model, ch, t, i, left)
    dm = O.alpha_dm(plan, B, Bidx, ket, bra, 0.0)
    m = 6
    a = G.predict_split(psi, model.phys, model.phys, offs, m, 1e-16, left, dm)
    b = G.split(psi, model.phys, model.phys, offs, m, 1e-16, left)
    assert a.bond == b.bond
    assert abs(a.truncated_weight - b.truncated_weight) <= 1e-12
    ta = G.twosite(a.A, a.B, p12, offs).data
    tb = G.twosite(b.A, b.B, p12, offs).data
    assert np.linalg.norm(ta - tb) <= 1e-12 * np.linalg.norm(tb)


def test_perturbed_sweeps_reach_exact_ground_energy():
    """Heisenberg L=10 from a bond-dimension-2 start: two-site sweeps with the
    perturbation (alpha 1e-3 for the first two sweeps, then 0, as the reference's
    alpha_initial / alpha_main / alpha_final schedule) reach the ED energy."""
    L = 10
    model = M.heisenberg(L)
    A = S.random_mps(model.phys, S.allowed_sectors(model.phys, L, model.total_charge, 2), np.random.default_rng(3))
    dm = G.TwoSiteDMRG(OracleBackend(), model, list(A), 32, jd_tol=1e-10, jd_maxiter=16,
                       alpha=lambda sweep: 1e-3 if sweep < 2 else 0.0)
    for sw in range(4):
        e = dm.sweep(sw)
    assert dm.log.phase_seconds.get("alpha_dm", 0.0) > 0.0
    assert abs(e - dense.ground_energy(model, L)) <= 1e-9


def test_perturbed_su2u1_sweeps_reach_fci():
    """SU2U1 quantum chemistry L=6 from a bond-dimension-3 start with the perturbation in
    the first two sweeps: the sweeps still reach the FCI singlet ground energy."""
    L, n = 6, 6
    h, eri = qc.synthetic_integrals(L)
    model = SU.quantum_chemistry(L, n, 0, h=h, eri=eri)
    A = S.random_mps(SU.PHYS, SU.allowed_sectors(L, (n, 0), 3), np.random.default_rng(2))
    dm = G.TwoSiteDMRG(OracleBackend(), model, list(A), 100, jd_tol=1e-10, jd_maxiter=12,
                       alpha=lambda sweep: 1e-3 if sweep < 2 else 0.0)
    for sw in range(4):
        e = dm.sweep(sw)
    assert dm.log.phase_seconds.get("alpha_dm", 0.0) > 0.0
    assert abs(e - dense.spin_sector_spectrum(h, eri, n, 0)[0]) <= 1e-9
