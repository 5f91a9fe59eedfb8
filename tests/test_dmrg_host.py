"""Host-side pieces of the sweep driver: two-site formation, SVD split and
right canonicalisation preserve the state (dense comparison on small chains)."""
import numpy as np
import pytest

import dense as D
from dmrgb200 import dmrg as G
from dmrgb200 import models as M
from dmrgb200 import mps as S


@pytest.mark.parametrize("name", ["heisenberg", "hubbard", "bose"])
def test_split_of_twosite_reproduces_state(name):
    L = 5
    model = {"heisenberg": M.heisenberg(L), "hubbard": M.fermi_hubbard(L, n_up=2, n_down=2),
             "bose": M.bose_hubbard(L, N=2)}[name]
    rng = np.random.default_rng(0)
    bonds = S.allowed_sectors(model.phys, L, model.total_charge, 6)
    A = S.random_mps(model.phys, bonds, rng)
    p12, offs = M.fuse_phys(model.phys, model.phys)
    psi = G.twosite(A[1], A[2], p12, offs)
    ref = D.mps_dense([t.dense() for t in A])
    for l2r in (True, False):
        res = G.split(psi, model.phys, model.phys, offs, 10 ** 6, 0.0, l2r)
        B = list(A)
        B[1], B[2] = res.A, res.B
        assert res.truncated_weight < 1e-12
        assert np.allclose(D.mps_dense([t.dense() for t in B]), ref, atol=1e-12)
    # two-site tensor matches the dense contraction of the pair
    core = D.twosite_dense(model.phys, model.phys, psi)
    pair = np.tensordot(A[1].dense(), A[2].dense(), axes=([2], [0]))
    assert np.allclose(core, pair, atol=1e-13)


def test_right_canonicalize_preserves_state_and_normalises():
    model = M.fermi_hubbard(6)
    rng = np.random.default_rng(1)
    bonds = S.allowed_sectors(model.phys, 6, model.total_charge, 8)
    A = S.random_mps(model.phys, bonds, rng)
    ref = D.mps_dense([t.dense() for t in A])
    B = G.right_canonicalize(A)
    got = D.mps_dense([t.dense() for t in B])
    assert np.allclose(got, ref / np.linalg.norm(ref), atol=1e-12)
    for t in B[1:]:
        Td = t.dense()
        X = Td.reshape(Td.shape[0], -1)
        assert np.allclose(X @ X.T, np.eye(X.shape[0]), atol=1e-12)


def test_left_canonicalize_preserves_state_and_normalises():
    model = M.fermi_hubbard(6, t=1.0, U=4.0)
    bonds = S.allowed_sectors(model.phys, 6, model.total_charge, 6)
    A = G.right_canonicalize(S.random_mps(model.phys, bonds, np.random.default_rng(4)))
    i = 3
    B = G.left_canonicalize(A, i)
    va, vb = D.mps_dense([t.dense() for t in A]), D.mps_dense([t.dense() for t in B])
    assert np.linalg.norm(va - vb) <= 1e-12 * np.linalg.norm(va)
    for t in B[:i]:
        Td = t.dense()
        X = Td.reshape(-1, Td.shape[2])
        assert np.allclose(X.T @ X, np.eye(X.shape[1]), atol=1e-12)
    for t in B[i + 1:]:
        Td = t.dense()
        X = Td.reshape(Td.shape[0], -1)
        assert np.allclose(X @ X.T, np.eye(X.shape[0]), atol=1e-12)


def test_truncation_keeps_largest_states():
    model = M.heisenberg(8)
    rng = np.random.default_rng(2)
    bonds = S.allowed_sectors(model.phys, 8, model.total_charge, 16)
    A = S.random_mps(model.phys, bonds, rng)
    p12, offs = M.fuse_phys(model.phys, model.phys)
    psi = G.twosite(A[3], A[4], p12, offs)
    res = G.split(psi, model.phys, model.phys, offs, 5, 0.0, True)
    assert sum(k for _, k in res.bond) == 5
    assert 0.0 < res.truncated_weight < 1.0


def _device_split_on_host(psi, phys, offs, m, cutoff, l2r):
    """The device split's host logic (DeviceSplitPlan) with the device work
    replaced by its host definitions: block copies by engine.apply_copies and the
    block SVDs by numpy, in the workspaces the device path uses."""
    from dmrgb200 import engine as E
    plan = G.DeviceSplitPlan(psi, phys, phys, offs)
    theta = np.zeros(max(plan.th_elems, 1))
    E.apply_copies(plan.gather, psi.data, theta)
    usv = np.zeros(max(plan.usv_elems, 1))
    for mc in plan.order:
        _, _, nr, nc, _ = plan.blocks[mc]
        k = min(nr, nc)
        t0 = plan.th_off[mc]
        U, sv, Vt = np.linalg.svd(theta[t0:t0 + nr * nc].reshape(nc, nr).T, full_matrices=False)
        usv[plan.u_off[mc]:plan.u_off[mc] + nr * k] = U.T.reshape(-1)
        usv[plan.vt_base + plan.vt_off[mc]:plan.vt_base + plan.vt_off[mc] + k * nc] = Vt.T.reshape(-1)
        usv[plan.s_base + plan.s_off[mc]:plan.s_base + plan.s_off[mc] + k] = sv
    kept, bond, tw = G._truncate(plan.svals(usv[plan.s_base:]), m, cutoff)
    A, B, lp, (a_lp, b0, end), copies = plan.scatter(kept, bond, psi.right, l2r)
    out = np.zeros(max(end, 1))
    E.apply_copies(copies, usv, out, usv)
    return A, B, out[:a_lp], out[a_lp:b0], out[b0:end], tw, bond


@pytest.mark.parametrize("name,m", [("heisenberg", 10 ** 6), ("hubbard", 10 ** 6), ("hubbard", 7), ("bose", 3)])
def test_device_split_plan_matches_host_split(name, m):
    """Gather, truncation and scatter of the device split reproduce the host
    split bitwise when the block SVDs agree (both numpy here)."""
    L = 5
    model = {"heisenberg": M.heisenberg(L), "hubbard": M.fermi_hubbard(L, n_up=2, n_down=2),
             "bose": M.bose_hubbard(L, N=2)}[name]
    rng = np.random.default_rng(3)
    bonds = S.allowed_sectors(model.phys, L, model.total_charge, 6)
    A = S.random_mps(model.phys, bonds, rng)
    p12, offs = M.fuse_phys(model.phys, model.phys)
    psi = G.twosite(A[1], A[2], p12, offs)
    for l2r in (True, False):
        ref = G.split(psi, model.phys, model.phys, offs, m, 1e-16, l2r)
        a, b, a_rp, a_lp, b_rp, tw, bond = _device_split_on_host(psi, model.phys, offs, m, 1e-16, l2r)
        assert bond == ref.bond and tw == ref.truncated_weight
        assert np.array_equal(a_rp, ref.A.data)
        assert np.array_equal(a_lp, ref.A.left_paired())
        assert np.array_equal(b_rp, ref.B.data)
