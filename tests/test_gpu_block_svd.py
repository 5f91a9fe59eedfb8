"""The two-site split on the device: dmrgb200_block_svd (one-sided Jacobi,
FP64) against numpy's LAPACK SVD, dmrgb200_copy_blocks against its host
definition, and split_device against the host split (svd / svd_truncate,
block_matrix/block_matrix_algorithms.h:95-113,185-298)."""
import numpy as np
import pytest

from dmrgb200 import _capi as capi
from dmrgb200 import dmrg as G
from dmrgb200 import engine as E
from dmrgb200 import models as M
from dmrgb200 import mps as S

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12

# shapes: tiny, odd, transposed, the shared-memory path and (past 200 KB of
# work) the global-scratch path
SHAPES = [(1, 1), (1, 7), (7, 1), (2, 2), (5, 3), (3, 5), (64, 64), (65, 33), (33, 65), (100, 100), (130, 130),
          (200, 120), (120, 200), (300, 17)]


def _svd_dev(mats):
    blocks, outs = [], []
    for a in mats:
        r, c = a.shape
        k = min(r, c)
        ad = torch.from_numpy(np.asfortranarray(a).reshape(-1, order="F").copy()).cuda()
        u = torch.full((max(r * k, 1),), np.nan, dtype=torch.float64, device="cuda")
        s = torch.full((max(k, 1),), np.nan, dtype=torch.float64, device="cuda")
        vt = torch.full((max(k * c, 1),), np.nan, dtype=torch.float64, device="cuda")
        blocks.append((r, c, ad, u, s, vt))
        outs.append((u, s, vt))
    E.block_svd(blocks)
    res = []
    for a, (u, s, vt) in zip(mats, outs):
        r, c = a.shape
        k = min(r, c)
        res.append((u.cpu().numpy()[:r * k].reshape(k, r).T, s.cpu().numpy()[:k], vt.cpu().numpy()[:k * c].reshape(c, k).T))
    return res


def _check(a, U, s, Vt):
    sref = np.linalg.svd(a, compute_uv=False)
    smax = max(sref[0] if sref.size else 0.0, 1e-300)
    assert np.all(np.diff(s) <= 0)
    assert np.max(np.abs(s - sref)) <= TOL * smax
    assert np.linalg.norm(U @ np.diag(s) @ Vt - a) <= TOL * max(np.linalg.norm(a), 1e-300)
    nz = s > 1e-13 * smax
    Un = U[:, nz]
    assert np.max(np.abs(Un.T @ Un - np.eye(Un.shape[1]))) <= TOL
    assert np.max(np.abs(Vt @ Vt.T - np.eye(Vt.shape[0]))) <= TOL


def test_block_svd_shapes_in_one_launch():
    rng = np.random.default_rng(0)
    mats = [rng.standard_normal(sh) for sh in SHAPES]
    for a, (U, s, Vt) in zip(mats, _svd_dev(mats)):
        _check(a, U, s, Vt)


def test_block_svd_graded_rank_deficient_and_zero_blocks():
    rng = np.random.default_rng(1)
    q1, _ = np.linalg.qr(rng.standard_normal((40, 40)))
    q2, _ = np.linalg.qr(rng.standard_normal((30, 30)))
    graded = q1[:, :30] @ np.diag(10.0 ** -np.linspace(0, 12, 30)) @ q2.T
    low = rng.standard_normal((40, 3)) @ rng.standard_normal((3, 30))
    zero = np.zeros((9, 4))
    mats = [graded, low, zero, 1e-200 * rng.standard_normal((6, 5)), 1e200 * rng.standard_normal((5, 6))]
    out = _svd_dev(mats)
    for a, (U, s, Vt) in zip(mats[:2], out[:2]):
        _check(a, U, s, Vt)
    assert np.all(out[2][1] == 0.0) and np.all(out[2][0] == 0.0)
    for a, (U, s, Vt) in zip(mats[3:], out[3:]):
        sref = np.linalg.svd(a, compute_uv=False)
        assert np.max(np.abs(s - sref)) <= TOL * sref[0]
        assert np.linalg.norm(U @ np.diag(s) @ Vt - a) <= TOL * np.linalg.norm(a)


def test_block_svd_rejects_null_blocks():
    rows = np.array([2], dtype=np.uint32)
    nul = (capi.C.c_void_p * 1)(None)
    st = capi.lib.dmrgb200_block_svd(1, capi.ptr(rows, capi.C.c_uint32), capi.ptr(rows, capi.C.c_uint32), nul, nul,
                                     nul, nul, None)
    assert st == 1


def test_copy_blocks_against_host_definition():
    rng = np.random.default_rng(2)
    src = rng.standard_normal(5000)
    scale = rng.standard_normal(64)
    recs, off = [], 0
    for k in range(40):
        r, c = int(rng.integers(0, 9)), int(rng.integers(0, 7))
        sl = r + int(rng.integers(0, 3))
        so = int(rng.integers(0, 5000 - max(sl, 1) * max(c, 1)))
        mode = int(rng.integers(0, 3))
        recs.append((so, sl, off, max(r, 1), r, c, mode, int(rng.integers(0, 40))))
        off += max(r, 1) * max(c, 1)
    cp = E.copy_records(recs)
    ref = np.zeros(off)
    E.apply_copies(cp, src, ref, scale)
    dst = torch.zeros(off, dtype=torch.float64, device="cuda")
    E.copy_blocks(cp, torch.from_numpy(src).cuda(), dst, torch.from_numpy(scale).cuda())
    torch.cuda.synchronize()
    assert np.array_equal(dst.cpu().numpy(), ref)


@pytest.mark.parametrize("name,m", [("hubbard", 10 ** 6), ("bose", 4), ("heisenberg", 10 ** 6)])
def test_split_device_matches_host_split(name, m):
    L = 6
    model = {"heisenberg": M.heisenberg(L), "hubbard": M.fermi_hubbard(L, n_up=3, n_down=3),
             "bose": M.bose_hubbard(L, N=3)}[name]
    rng = np.random.default_rng(5)
    bonds = S.allowed_sectors(model.phys, L, model.total_charge, 12)
    A = S.random_mps(model.phys, bonds, rng)
    p12, offs = M.fuse_phys(model.phys, model.phys)
    psi = G.twosite(A[2], A[3], p12, offs)
    psi_dev = E.to_device(psi.data)
    for l2r in (True, False):
        ref = G.split(psi, model.phys, model.phys, offs, m, 1e-16, l2r)
        got = G.split_device(psi_dev, psi, model.phys, model.phys, offs, m, 1e-16, l2r)
        assert got.bond == ref.bond
        assert abs(got.truncated_weight - ref.truncated_weight) <= 1e-12
        # the kept two-site tensor is gauge independent
        t_ref = G.twosite(ref.A, ref.B, p12, offs).data
        t_got = G.twosite(got.A, got.B, p12, offs).data
        assert np.linalg.norm(t_got - t_ref) <= TOL * np.linalg.norm(t_ref)
        # device copies agree with the host copies; A left-normalised (l2r) or B right-normalised
        assert np.array_equal(got.dev_A.cpu().numpy(), got.A.data)
        assert np.array_equal(got.dev_A_lp.cpu().numpy(), got.A.left_paired())
        assert np.array_equal(got.dev_B.cpu().numpy(), got.B.data)
        if l2r:
            lp = S.left_paired_layout(got.A.phys, got.A.left, got.A.right)
            for rb in range(len(got.A.right)):
                X = S.block_view(got.A.left_paired(), lp, rb)
                assert np.max(np.abs(X.T @ X - np.eye(X.shape[1]))) <= TOL
        else:
            for lb in range(len(got.B.left)):
                X = S.block_view(got.B.data, got.B.rp, lb)
                assert np.max(np.abs(X @ X.T - np.eye(X.shape[0]))) <= TOL
