"""Two-site DMRG sweeps driving the device hot path.

The optimizer mirrors the reference's ts_optimize::sweep
(dmrg/framework/dmrg/optimize/ts_optimize.hpp:114-362) and its boundary caches
(optimize/optimize.h:71-195): for every site pair the two-site tensor is
formed, its lowest eigenpair is found by Jacobi-Davidson on the device
(dmrgb200_solve over a dmrgb200 H·psi plan), the result is split by a
block-wise SVD truncated to the bond dimension, and the left (right) boundary
is advanced by a device boundary step.  The SVD split and the two-site tensor
formation run on the host in FP64 (numpy/LAPACK).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi
from . import engine as E
from . import models as M
from . import mps as S


def _sub(t: S.SiteTensor, lb, s, ss):
    r0, c0, ml, mr, rb = t.rp.sub[(lb, s, ss)]
    return S.block_view(t.data, t.rp, lb)[:, c0:c0 + mr], rb


def twosite(A: S.SiteTensor, B: S.SiteTensor, p12, offs) -> S.SiteTensor:
    """psi = A . B over the shared bond, physical index fused (TwoSiteTensor,
    mp_tensors/twositetensor.hpp:28-43)."""
    psi = S.SiteTensor(p12, A.left, B.right)
    p12pos = {c: k for k, (c, _) in enumerate(p12)}
    d1 = dict(A.phys)
    d2 = dict(B.phys)
    for (lb, s1, i1), (_, c0a, ml, mm, mb) in A.rp.sub.items():
        a = S.block_view(A.data, A.rp, lb)[:, c0a:c0a + mm]
        c1 = A.phys[s1][0]
        for s2, (c2, dd2) in enumerate(B.phys):
            for i2 in range(dd2):
                key = (mb, s2, i2)
                if key not in B.rp.sub:
                    continue
                b, rb = _sub(B, mb, s2, i2)
                f = (c1[0] + c2[0], c1[1] + c2[1])
                ss = offs[(c1, c2)] + i1 * d2[c2] + i2
                k = (lb, p12pos[f], ss)
                if k not in psi.rp.sub:
                    continue
                _, c0, _, mr, _ = psi.rp.sub[k]
                S.block_view(psi.data, psi.rp, lb)[:, c0:c0 + mr] += a @ b
    del d1
    return psi


@dataclass
class SplitResult:
    A: S.SiteTensor
    B: S.SiteTensor
    truncated_weight: float
    bond: list
    # device copies written by split_device: A right-paired, A left-paired, B right-paired
    dev_A: object = None
    dev_A_lp: object = None
    dev_B: object = None


def _mid_blocks(psi: S.SiteTensor, phys1, phys2, offs):
    """Rows (s1, i1, lc, ml) and columns (s2, i2, rc, mr) of the matrix Theta of
    every middle charge, and the psi sub-blocks that fill it as (row offset,
    column offset, ml, mr, psi block, column in that block) (the reshape of
    TwoSiteTensor to a left-paired matrix, mp_tensors/twositetensor.hpp:153-200)."""
    left, right = psi.left, psi.right
    lpos = {c: i for i, (c, _) in enumerate(left)}
    rpos = {c: i for i, (c, _) in enumerate(right)}
    p12pos = {c: k for k, (c, _) in enumerate(psi.phys)}
    mids = {}
    for s1, (c1, d1) in enumerate(phys1):
        for lc, ml in left:
            mc = (lc[0] + c1[0], lc[1] + c1[1])
            for i1 in range(d1):
                mids.setdefault(mc, [[], []])[0].append((s1, i1, lc, ml))
    for mc in list(mids):
        for s2, (c2, d2) in enumerate(phys2):
            rc = (mc[0] + c2[0], mc[1] + c2[1])
            if rc not in rpos:
                continue
            for i2 in range(d2):
                mids[mc][1].append((s2, i2, rc, right[rpos[rc]][1]))
    d2s = dict(phys2)
    out = {}
    for mc, (rows, cols) in mids.items():
        nr, nc = sum(r[3] for r in rows), sum(c[3] for c in cols)
        if nr == 0 or nc == 0:
            continue
        fills = []
        ro = 0
        for (s1, i1, lc, ml) in rows:
            co = 0
            c1 = phys1[s1][0]
            for (s2, i2, rc, mr) in cols:
                c2 = phys2[s2][0]
                f = (c1[0] + c2[0], c1[1] + c2[1])
                k = (lpos[lc], p12pos[f], offs[(c1, c2)] + i1 * d2s[c2] + i2)
                if k in psi.rp.sub:
                    fills.append((ro, co, ml, mr, lpos[lc], psi.rp.sub[k][1]))
                co += mr
            ro += ml
        out[mc] = (rows, cols, nr, nc, fills)
    return out


def _truncate(svals: dict, m: int, cutoff: float):
    """Kept states per middle charge: the m largest singular values over all
    blocks above cutoff times the largest (svd_truncate,
    block_matrix/block_matrix_algorithms.h:185-298).  Returns (kept, bond,
    truncated weight)."""
    allsv = np.concatenate([v for v in svals.values()]) if svals else np.zeros(0)
    total = float(np.sum(allsv ** 2))
    order = np.sort(allsv)[::-1]
    keep_n = min(m, int(np.sum(order > cutoff * (order[0] if order.size else 0))))
    thresh = order[keep_n - 1] if keep_n > 0 else np.inf
    kept = {}
    count = 0
    for mc in sorted(svals):
        sv = svals[mc]
        k = int(np.sum(sv >= thresh))
        k = min(k, keep_n - count)
        if k > 0:
            kept[mc] = k
            count += k
    bond = [(mc, kept[mc]) for mc in sorted(kept)]
    tw = 1.0 - float(sum(np.sum(svals[mc][:kept[mc]] ** 2) for mc in kept)) / total if total > 0 else 0.0
    return kept, bond, tw


def split(psi: S.SiteTensor, phys1, phys2, offs, m: int, cutoff: float, left_to_right: bool) -> SplitResult:
    """SVD split of a two-site tensor with truncation to m states and relative
    cutoff (svd_truncate, block_matrix/block_matrix_algorithms.h:185-298):
    left-to-right keeps U left-normalised and moves S V^T right, right-to-left
    keeps V^T right-normalised and moves U S left.  Host (numpy) SVDs."""
    left, right = psi.left, psi.right
    lpos = {c: i for i, (c, _) in enumerate(left)}
    svds = {}
    for mc, (rows, cols, nr, nc, fills) in _mid_blocks(psi, phys1, phys2, offs).items():
        Th = np.zeros((nr, nc))
        for (ro, co, ml, mr, lb, c0) in fills:
            Th[ro:ro + ml, co:co + mr] = S.block_view(psi.data, psi.rp, lb)[:, c0:c0 + mr]
        U, sv, Vt = np.linalg.svd(Th, full_matrices=False)
        svds[mc] = (U, sv, Vt, rows, cols)
    kept, bond, tw = _truncate({mc: v[1] for mc, v in svds.items()}, m, cutoff)
    A = S.SiteTensor(phys1, left, bond)
    B = S.SiteTensor(phys2, bond, right)
    bpos = {c: i for i, (c, _) in enumerate(bond)}
    for mc, k in kept.items():
        U, sv, Vt, rows, cols = svds[mc]
        if left_to_right:
            Uk, Vk = U[:, :k], sv[:k, None] * Vt[:k, :]
        else:
            Uk, Vk = U[:, :k] * sv[None, :k], Vt[:k, :]
        ro = 0
        for (s1, i1, lc, ml) in rows:
            key = (lpos[lc], s1, i1)
            if key in A.rp.sub:
                _, c0, _, mr, rb = A.rp.sub[key]
                assert rb == bpos[mc]
                S.block_view(A.data, A.rp, lpos[lc])[:, c0:c0 + mr] = Uk[ro:ro + ml, :]
            ro += ml
        co = 0
        for (s2, i2, rc, mr) in cols:
            key = (bpos[mc], s2, i2)
            _, c0, _, _, _ = B.rp.sub[key]
            S.block_view(B.data, B.rp, bpos[mc])[:, c0:c0 + mr] = Vk[:, co:co + mr]
            co += mr
    return SplitResult(A, B, tw, bond)


def theta_site(psi: S.SiteTensor, phys1, phys2, offs, left_to_right: bool):
    """The two-site tensor viewed as one site tensor, as the state prediction of the
    reference does (prediction.hpp:152-171 / 193-212): left-to-right, the tensor at
    site 1 whose right bond is the middle index (one block per middle charge, the
    columns of Theta); right-to-left, the tensor at site 2 whose left bond is the
    middle index (the rows of Theta).  Its left-paired (right-paired) block of a
    middle charge is Theta of that charge.  Returns (tensor, middle blocks)."""
    mids = _mid_blocks(psi, phys1, phys2, offs)
    order = sorted(mids)
    if left_to_right:
        t = S.SiteTensor(phys1, psi.left, [(mc, mids[mc][3]) for mc in order])
    else:
        t = S.SiteTensor(phys2, [(mc, mids[mc][2]) for mc in order], psi.right)
    lpos = {c: i for i, (c, _) in enumerate(psi.left)}
    for b, mc in enumerate(order):
        rows, cols, nr, nc, fills = mids[mc]
        Th = np.zeros((nr, nc))
        for (ro, co, ml, mr, lb, c0) in fills:
            Th[ro:ro + ml, co:co + mr] = S.block_view(psi.data, psi.rp, lb)[:, c0:c0 + mr]
        if left_to_right:
            ro = 0
            for (s1, i1, lc, ml) in rows:
                key = (lpos[lc], s1, i1)
                if key in t.rp.sub:
                    _, c0, _, mr, rb = t.rp.sub[key]
                    S.block_view(t.data, t.rp, lpos[lc])[:, c0:c0 + mr] = Th[ro:ro + ml, :]
                ro += ml
        else:
            co = 0
            for (s2, i2, rc, mr) in cols:
                _, c0, _, _, _ = t.rp.sub[(b, s2, i2)]
                S.block_view(t.data, t.rp, b)[:, c0:c0 + mr] = Th[:, co:co + mr]
                co += mr
    return t, mids


def predict_split(psi: S.SiteTensor, phys1, phys2, offs, m: int, cutoff: float, left_to_right: bool, dm_blocks):
    """Two-site split with the reference's state prediction (predict_split_l2r / r2l,
    prediction.hpp:152-240): the density matrix of every middle charge is
    Theta Theta^T (left-to-right; Theta^T Theta right-to-left) plus alpha times the
    perturbation terms, as dm_blocks (the backend's alpha_dm on theta_site) returns
    them in middle-charge order; it is diagonalised on the host (eigh), truncated like
    heev_truncate (block_matrix_algorithms.h:298-346: the square roots of the
    eigenvalues as singular values, svd truncation rules), and left-to-right keeps the
    eigenvectors U as site 1 and U^T Theta as site 2, right-to-left U^T as site 2 and
    Theta U as site 1."""
    mids = _mid_blocks(psi, phys1, phys2, offs)
    order = sorted(mids)
    eig = {}
    for b, mc in enumerate(order):
        w, U = np.linalg.eigh(0.5 * (dm_blocks[b] + dm_blocks[b].T))
        w, U = w[::-1], U[:, ::-1]
        eig[mc] = (np.sqrt(np.maximum(w, 0.0)), U)
    kept, bond, tw = _truncate({mc: v[0] for mc, v in eig.items()}, m, cutoff)
    left, right = psi.left, psi.right
    lpos = {c: i for i, (c, _) in enumerate(left)}
    A = S.SiteTensor(phys1, left, bond)
    B = S.SiteTensor(phys2, bond, right)
    bpos = {c: i for i, (c, _) in enumerate(bond)}
    for mc, k in kept.items():
        rows, cols, nr, nc, fills = mids[mc]
        Th = np.zeros((nr, nc))
        for (ro, co, ml, mr, lb, c0) in fills:
            Th[ro:ro + ml, co:co + mr] = S.block_view(psi.data, psi.rp, lb)[:, c0:c0 + mr]
        Uk = eig[mc][1][:, :k]
        if left_to_right:
            Ak, Bk = Uk, Uk.T @ Th
        else:
            Ak, Bk = Th @ Uk, Uk.T
        ro = 0
        for (s1, i1, lc, ml) in rows:
            key = (lpos[lc], s1, i1)
            if key in A.rp.sub:
                _, c0, _, mr, rb = A.rp.sub[key]
                S.block_view(A.data, A.rp, lpos[lc])[:, c0:c0 + mr] = Ak[ro:ro + ml, :]
            ro += ml
        co = 0
        for (s2, i2, rc, mr) in cols:
            _, c0, _, _, _ = B.rp.sub[(bpos[mc], s2, i2)]
            S.block_view(B.data, B.rp, bpos[mc])[:, c0:c0 + mr] = Bk[:, co:co + mr]
            co += mr
    return SplitResult(A, B, tw, bond)


class DeviceSplitPlan:
    """Host-side part of the device split: the layout of Theta, U, s and V^T in
    device workspaces and the gather copies from psi (no device work here)."""

    def __init__(self, psi: S.SiteTensor, phys1, phys2, offs):
        self.psi, self.phys1, self.phys2 = psi, phys1, phys2
        self.blocks = _mid_blocks(psi, phys1, phys2, offs)
        self.order = sorted(self.blocks)
        self.th_off, self.u_off, self.s_off, self.vt_off = {}, {}, {}, {}
        th = u = sv = vt = 0
        for mc in self.order:
            _, _, nr, nc, _ = self.blocks[mc]
            k = min(nr, nc)
            self.th_off[mc], self.u_off[mc], self.s_off[mc], self.vt_off[mc] = th, u, sv, vt
            th += nr * nc
            u += nr * k
            sv += k
            vt += k * nc
        self.th_elems = th
        # one workspace for U | V^T | s
        self.vt_base, self.s_base = u, u + vt
        self.usv_elems = u + vt + sv
        rp = psi.rp
        rec = []
        for mc in self.order:
            _, _, nr, nc, fills = self.blocks[mc]
            for (ro, co, ml, mr, lb, c0) in fills:
                rec.append((rp.offs[lb] + c0 * rp.rows[lb], rp.rows[lb], self.th_off[mc] + ro + co * nr, nr, ml, mr,
                            0, 0))
        self.gather = E.copy_records(rec)

    def svals(self, s_host: np.ndarray) -> dict:
        out = {}
        for mc in self.order:
            _, _, nr, nc, _ = self.blocks[mc]
            o = self.s_off[mc]
            out[mc] = s_host[o:o + min(nr, nc)]
        return out

    def scatter(self, kept: dict, bond, right, left_to_right: bool):
        """Site tensors of the new bond and the copies that fill them from the
        U | V^T | s workspace: A right-paired at 0, A left-paired at a_lp, B
        right-paired at b0 of one output buffer."""
        psi, phys1, phys2 = self.psi, self.phys1, self.phys2
        A = S.SiteTensor(phys1, psi.left, bond)
        B = S.SiteTensor(phys2, bond, right)
        lp = S.left_paired_layout(phys1, psi.left, bond)
        a_lp, b0 = A.rp.total, A.rp.total + lp.total
        lpos = {c: i for i, (c, _) in enumerate(psi.left)}
        bpos = {c: i for i, (c, _) in enumerate(bond)}
        u_mode = capi.SCALE_NONE if left_to_right else capi.SCALE_COLS
        vt_mode = capi.SCALE_ROWS if left_to_right else capi.SCALE_NONE
        rec = []
        for mc, k in kept.items():
            rows, cols, nr, nc, _ = self.blocks[mc]
            k0 = min(nr, nc)
            uo, so, vo = self.u_off[mc], self.s_base + self.s_off[mc], self.vt_base + self.vt_off[mc]
            rb = bpos[mc]
            ro = 0
            for (s1, i1, lc, ml) in rows:
                key = (lpos[lc], s1, i1)
                if key in A.rp.sub:
                    lb = lpos[lc]
                    c0 = A.rp.sub[key][1]
                    rec.append((uo + ro, nr, A.rp.offs[lb] + c0 * A.rp.rows[lb], A.rp.rows[lb], ml, k, u_mode, so))
                    r0 = lp.sub[(rb, s1, i1)][0]
                    rec.append((uo + ro, nr, a_lp + lp.offs[rb] + r0, lp.rows[rb], ml, k, u_mode, so))
                ro += ml
            co = 0
            for (s2, i2, rc, mr) in cols:
                c0 = B.rp.sub[(rb, s2, i2)][1]
                rec.append((vo + co * k0, k0, b0 + B.rp.offs[rb] + c0 * B.rp.rows[rb], B.rp.rows[rb], k, mr, vt_mode,
                            so))
                co += mr
        return A, B, lp, (a_lp, b0, b0 + B.rp.total), E.copy_records(rec)


def split_device(psi_dev, psi: S.SiteTensor, phys1, phys2, offs, m: int, cutoff: float, left_to_right: bool,
                 device: int = 0) -> SplitResult:
    """The split of `split` with the two-site tensor on the device: Theta is
    gathered from psi_dev, every block is decomposed by dmrgb200_block_svd, the
    singular values alone come to the host for the truncation choice, and U,
    S V^T (or U S, V^T) are scattered into the new site tensors on the device.
    The site tensors are also copied to the host (SplitResult.A / .B)."""
    import torch
    plan = DeviceSplitPlan(psi, phys1, phys2, offs)
    dev = psi_dev.device
    sh = torch.cuda.current_stream(dev).cuda_stream  # every step of the split on torch's current stream
    theta = torch.zeros(max(plan.th_elems, 1), dtype=torch.float64, device=dev)
    E.copy_blocks(plan.gather, psi_dev, theta, stream=sh)
    usv = torch.empty(max(plan.usv_elems, 1), dtype=torch.float64, device=dev)
    blocks = []
    for mc in plan.order:
        _, _, nr, nc, _ = plan.blocks[mc]
        k = min(nr, nc)
        t0, u0, s0, v0 = plan.th_off[mc], plan.u_off[mc], plan.s_base + plan.s_off[mc], plan.vt_base + plan.vt_off[mc]
        blocks.append((nr, nc, theta[t0:t0 + nr * nc], usv[u0:u0 + nr * k], usv[s0:s0 + k], usv[v0:v0 + k * nc]))
    E.block_svd(blocks, sh)
    s_host = usv[plan.s_base:plan.s_base + (plan.usv_elems - plan.s_base)].cpu().numpy()
    kept, bond, tw = _truncate(plan.svals(s_host), m, cutoff)
    A, B, lp, (a_lp, b0, end), copies = plan.scatter(kept, bond, psi.right, left_to_right)
    out = torch.zeros(max(end, 1), dtype=torch.float64, device=dev)
    E.copy_blocks(copies, usv, out, usv, stream=sh)
    host = out.cpu().numpy()
    A.data = host[:a_lp].copy()
    B.data = host[b0:end].copy()
    return SplitResult(A, B, tw, bond, dev_A=out[:a_lp], dev_A_lp=out[a_lp:b0], dev_B=out[b0:end])


def right_canonicalize(tensors, cutoff: float = 1e-14):
    """Make sites 1..L-1 right-normalised by per-charge SVDs, absorbing the
    remainder into the left neighbour.  Singular vectors whose singular value is at
    most `cutoff` times the block's largest are dropped; cutoff = 0 keeps every
    block at full rank (the singular vectors stay orthonormal however small their
    weight), so the bond dimensions of a synthetic environment survive the products
    of positive random blocks, whose spectra decay by orders of magnitude per site."""
    out = list(tensors)
    for j in range(len(out) - 1, 0, -1):
        t = out[j]
        new_left, Vs, absorb = [], {}, {}
        for lb, (lc, ml) in enumerate(t.left):
            blk = S.block_view(t.data, t.rp, lb)
            if blk.size == 0:
                continue
            U, sv, Vt = np.linalg.svd(blk, full_matrices=False)
            k = int(np.sum(sv > cutoff * max(sv[0], 1e-300))) if sv.size else 0
            if k == 0:
                continue
            new_left.append((lc, k))
            Vs[lc] = Vt[:k]
            absorb[lc] = U[:, :k] * sv[None, :k]
        nt = S.SiteTensor(t.phys, new_left, t.right)
        for lb, (lc, k) in enumerate(new_left):
            S.block_view(nt.data, nt.rp, lb)[:, :] = Vs[lc]
        prev = out[j - 1]
        np_ = S.SiteTensor(prev.phys, prev.left, new_left)
        npos = {c: i for i, (c, _) in enumerate(new_left)}
        for (lb, s, ss), (_, c0, ml, mr, rb) in prev.rp.sub.items():
            mc = prev.right[rb][0]
            if mc not in npos:
                continue
            key = (lb, s, ss)
            _, c1, _, k, _ = np_.rp.sub[key]
            S.block_view(np_.data, np_.rp, lb)[:, c1:c1 + k] = \
                S.block_view(prev.data, prev.rp, lb)[:, c0:c0 + mr] @ absorb[mc]
        out[j] = nt
        out[j - 1] = np_
    n = out[0].norm()
    out[0].data /= n
    return out


def left_canonicalize(tensors, upto: int, cutoff: float = 1e-14):
    """Make sites 0..upto-1 left-normalised by per-charge SVDs of their
    left-paired blocks, absorbing S V^T into the right neighbour (the mirror of
    right_canonicalize); bond dimensions drop only where a block is rank
    deficient (by `cutoff`, as in right_canonicalize).  Returns the new tensor list."""
    out = list(tensors)
    for j in range(upto):
        t, nxt = out[j], out[j + 1]
        lp = S.left_paired_layout(t.phys, t.left, t.right)
        lpd = t.left_paired()
        new_right, Us, absorb = [], {}, {}
        for rb, (rc, mr) in enumerate(t.right):
            blk = S.block_view(lpd, lp, rb)
            if blk.size == 0:
                continue
            U, sv, Vt = np.linalg.svd(blk, full_matrices=False)
            k = int(np.sum(sv > cutoff * max(sv[0], 1e-300))) if sv.size else 0
            if k == 0:
                continue
            new_right.append((rc, k))
            Us[rc] = U[:, :k]
            absorb[rc] = sv[:k, None] * Vt[:k]
        nt = S.SiteTensor(t.phys, t.left, new_right)
        nlp = S.left_paired_layout(t.phys, t.left, new_right)
        for (rb, s, ss), (r0, _, ml, k, lb) in nlp.sub.items():
            rc = new_right[rb][0]
            _, c0, _, _, _ = nt.rp.sub[(lb, s, ss)]
            S.block_view(nt.data, nt.rp, lb)[:, c0:c0 + k] = Us[rc][r0:r0 + ml, :]
        nn = S.SiteTensor(nxt.phys, new_right, nxt.right)
        npos = {c: i for i, (c, _) in enumerate(new_right)}
        for (lb, s, ss), (_, c0, ml, mr, rb) in nxt.rp.sub.items():
            lc = nxt.left[lb][0]
            if lc not in npos:
                continue
            nlb = npos[lc]
            _, c1, _, _, _ = nn.rp.sub[(nlb, s, ss)]
            S.block_view(nn.data, nn.rp, nlb)[:, c1:c1 + mr] = absorb[lc] @ S.block_view(nxt.data, nxt.rp, lb)[:, c0:c0 + mr]
        out[j], out[j + 1] = nt, nn
    return out


@dataclass
class SweepLog:
    energies: list = field(default_factory=list)      # (sweep, site, energy, iterations, truncated weight)
    sweep_seconds: list = field(default_factory=list)
    hpsi_calls: int = 0
    solve_ms: float = 0.0   # device time of the eigen-solves
    phase_seconds: dict = field(default_factory=dict)  # host wall time per phase of the site steps


class DeviceBackend:
    """Hot-path operations on the device through libdmrgb200: boundary steps,
    H·psi plans and the Jacobi-Davidson solver (dmrgb200_solve)."""

    def __init__(self, ctx: E.Context, precision: int = capi.PREC_FP64, slices: int | None = None,
                 slice_target: float = 1e-10, reuse_plans: bool = True):
        """precision: of the H·psi inside every solve (capi.PREC_FP64 or capi.PREC_FP64_EMULATED:
        contractions on the INT8 tensor cores, orthogonalisation, Rayleigh-Ritz and energies in
        FP64).  Emulated solves use `slices` digit planes, or, with slices None, the smallest
        count whose H·psi of the start vector is within slice_target of FP64 (tuned per site
        problem, dmrgb200_plan_tune_slices)."""
        import torch
        self.torch, self.ctx = torch, ctx
        self.precision, self.slices, self.slice_target = precision, slices, slice_target
        # reuse_plans: one cached (schedule, device plan, output buffer) per site and kind,
        # reused while the site's bond sectors and input boundary stay the same -- in the
        # sweeps after the bond dimensions have settled every schedule, lowered step
        # program and captured solver graph is reused (the reference rebuilds its
        # schedules at every site of every sweep, site_hamil_schedule.hpp:40-93)
        self.reuse_plans = reuse_plans
        self.cache = {}
        # schedules by structure: (kind, MPO tensor, bond sectors, boundary index signatures); a
        # schedule depends on nothing else, so after the bond sectors settle every later sweep
        # finds its schedules here even though its boundary buffers and index objects are new
        self.schedules = {}
        self.schedule_hits = 0
        self.cache_hits = 0
        self.cache_misses = 0
        self.slices_used = []  # (digit planes, relative H·psi error of the start vector) per emulated solve
        # host seconds per phase of the site problems (schedule building, plan lowering, solve)
        self.phase_seconds = {"schedule": 0.0, "plan": 0.0, "solve": 0.0}

    def edge(self, symm, index):
        idx = E.edge_bindex(symm, index)
        return idx, E.to_device(idx.edge_values(), self.ctx.device)

    def _step(self, left, model, W, idx, buf, t: S.SiteTensor, dev_rp=None, dev_lp=None):
        """One boundary step; dev_rp / dev_lp are device copies of t (right- and
        left-paired) when the split left them on the device."""
        dev = self.ctx.device
        t0 = time.perf_counter()
        site_key = ("L" if left else "R", id(W))
        full_key = (id(idx), buf.data_ptr(), tuple(t.left), tuple(t.right))
        hit = self.cache.get(site_key) if self.reuse_plans else None
        if hit is not None and hit[0] == full_key:
            _, idx_keep, nidx, plan, out = hit
            self.cache_hits += 1
        else:
            skey = (site_key, tuple(t.left), tuple(t.right), idx.signature())
            cached = self.schedules.get(skey) if self.reuse_plans else None
            if cached is not None:
                sched, nidx = cached[1], cached[2]
                self.schedule_hits += 1
            elif left:
                sched, nidx = E.schedule_left_step(model.phys, t.left, t.right, W, idx, True)
            else:
                sched, nidx = E.schedule_right_step(model.phys, t.left, t.right, W, idx, True)
            if self.reuse_plans and cached is None:
                self.schedules[skey] = (W, sched, nidx)  # W kept alive: its id is part of the key
            if left:
                plan = E.DevicePlan(self.ctx, sched.plan, left_addr=idx.cohort_addresses(buf.data_ptr()))
            else:
                plan = E.DevicePlan(self.ctx, sched.plan, other_addr=idx.cohort_addresses(buf.data_ptr()))
            out = self.torch.zeros(max(nidx.n_elems, 1), dtype=self.torch.float64, device=buf.device)
            self.cache_misses += 1
            if self.reuse_plans:
                # idx is kept alive with the entry, so its id cannot be reused by another index
                self.cache[site_key] = (full_key, idx, nidx, plan, out)
        if left:
            ket = dev_rp if dev_rp is not None else E.to_device(t.data, dev)
            bra = dev_lp if dev_lp is not None else E.to_device(t.left_paired(), dev)
        else:
            ket = bra = dev_rp if dev_rp is not None else E.to_device(t.data, dev)
        t1 = time.perf_counter()
        plan.step(ket.data_ptr(), bra.data_ptr(), nidx.cohort_addresses(out.data_ptr()))
        t2 = time.perf_counter()
        if not self.reuse_plans:
            del plan
        t3 = time.perf_counter()
        ph = self.phase_seconds
        ph["step_schedule"] = ph.get("step_schedule", 0.0) + t1 - t0
        ph["step_execute"] = ph.get("step_execute", 0.0) + t2 - t1
        ph["step_destroy"] = ph.get("step_destroy", 0.0) + t3 - t2
        return nidx, out

    def left_step(self, model, W, Lidx, Lbuf, t: S.SiteTensor, dev_rp=None, dev_lp=None):
        return self._step(True, model, W, Lidx, Lbuf, t, dev_rp, dev_lp)

    def right_step(self, model, W, Ridx, Rbuf, t: S.SiteTensor, dev_rp=None):
        return self._step(False, model, W, Ridx, Rbuf, t, dev_rp)

    def galpha(self, plan: dict, Lidx, Lbuf, Ridx, Rbuf, x: np.ndarray) -> np.ndarray:
        """d<x|H_eff x>/d alpha per plan term (dmrgb200_hpsi_adjoint on the device)."""
        dp = E.DevicePlan(self.ctx, plan, left_addr=Lidx.cohort_addresses(Lbuf.data_ptr()),
                          other_addr=Ridx.cohort_addresses(Rbuf.data_ptr()))
        xd = E.to_device(x, self.ctx.device)
        ga = self.torch.empty(max(len(plan["term_alpha"]), 1), dtype=self.torch.float64, device=xd.device)
        dp.adjoint(xd.data_ptr(), xd.data_ptr(), 0, ga.data_ptr())
        return ga.cpu().numpy()[:len(plan["term_alpha"])]

    def alpha_dm(self, phys, W, idx, buf, t: S.SiteTensor, alpha: float, left: bool):
        """Density-matrix blocks (host, per bra block of the step) of the split with the
        perturbation, for t = theta_site(...): dmrgb200_step_alpha_dm on a step plan
        without boundary skipping (alpha_dm_direct builds its schedule with skip off,
        move_boundary.hpp:72-75 / 126-129)."""
        dev = self.ctx.device
        if left:
            sched, _ = E.schedule_left_step(phys, t.left, t.right, W, idx, False)
            plan = E.DevicePlan(self.ctx, sched.plan, left_addr=idx.cohort_addresses(buf.data_ptr()))
            ket, bra = E.to_device(t.data, dev), E.to_device(t.left_paired(), dev)
            dims = [int(r) for r in sched.plan["out_rows"]]
        else:
            sched, _ = E.schedule_right_step(phys, t.left, t.right, W, idx, False)
            plan = E.DevicePlan(self.ctx, sched.plan, other_addr=idx.cohort_addresses(buf.data_ptr()))
            ket = bra = E.to_device(t.data, dev)
            dims = [int(c) for c in sched.plan["out_cols"]]
        offs = np.concatenate([[0], np.cumsum([d * d for d in dims])]).astype(np.int64)
        store = self.torch.zeros(max(int(offs[-1]), 1), dtype=self.torch.float64, device=buf.device)
        addr = np.array([store.data_ptr() + 8 * int(o) for o in offs[:-1]], dtype=np.uint64)
        plan.alpha_dm(ket.data_ptr(), bra.data_ptr(), addr, alpha)
        flat = store.cpu().numpy()
        return [flat[offs[b]:offs[b + 1]].reshape(d, d, order="F") for b, d in enumerate(dims)]

    def solve(self, p12, psi: S.SiteTensor, W12, Lidx, Lbuf, Ridx, Rbuf, tol, max_iter, keep_on_device=False):
        """Lowest eigenpair of the site problem; the eigenvector comes back as a
        host array, or as the device tensor with keep_on_device."""
        t0 = time.perf_counter()
        site_key = ("H", id(W12))
        full_key = (id(Lidx), id(Ridx), Lbuf.data_ptr(), Rbuf.data_ptr(), tuple(psi.left), tuple(psi.right))
        hit = self.cache.get(site_key) if self.reuse_plans else None
        if hit is not None and hit[0] == full_key:
            plan = hit[3]
            plan.boundaries_changed()  # the bound boundary buffers were rewritten since its last solve
            self.cache_hits += 1
            t1 = t2 = time.perf_counter()
        else:
            skey = (site_key, tuple(psi.left), tuple(psi.right), Lidx.signature(), Ridx.signature())
            cached = self.schedules.get(skey) if self.reuse_plans else None
            if cached is not None:
                sched = cached[1]
                self.schedule_hits += 1
            else:
                sched = E.schedule_hpsi(p12, psi.left, psi.right, W12, Lidx, Ridx)
                if self.reuse_plans:
                    self.schedules[skey] = (W12, sched)
            t1 = time.perf_counter()
            plan = E.DevicePlan(self.ctx, sched.plan, left_addr=Lidx.cohort_addresses(Lbuf.data_ptr()),
                                other_addr=Ridx.cohort_addresses(Rbuf.data_ptr()))
            t2 = time.perf_counter()
            self.cache_misses += 1
            if self.reuse_plans:
                self.cache[site_key] = (full_key, Lidx, Ridx, plan)
        xd = E.to_device(psi.data, self.ctx.device)
        xo = self.torch.zeros_like(xd)
        if self.precision == capi.PREC_FP64_EMULATED and not getattr(plan, "emulation_set", False):
            # once per plan: a reused plan keeps its slice count (and its captured solver graph)
            if self.slices is None:
                self.slices_used.append(plan.tune_slices(xd.data_ptr(), self.slice_target))
            else:
                plan.set_slices(self.slices)
            plan.set_precision(capi.PREC_FP64_EMULATED)
            plan.emulation_set = True
        energy, st = plan.solve(xd.data_ptr(), xo.data_ptr(), xd.numel(), tol=tol, max_iter=max_iter)
        out = xo if keep_on_device else xo.cpu().numpy()
        t3 = time.perf_counter()
        if not self.reuse_plans:
            del plan
        t4 = time.perf_counter()
        self.phase_seconds["schedule"] += t1 - t0
        self.phase_seconds["plan"] += t2 - t1
        self.phase_seconds["solve"] += t3 - t2
        self.phase_seconds["plan_destroy"] = self.phase_seconds.get("plan_destroy", 0.0) + t4 - t3
        return energy, out, st.iterations, st.solve_ms

    def sync(self):
        self.torch.cuda.synchronize(self.ctx.device)


class TwoSiteDMRG:
    def __init__(self, backend, model: M.Model, tensors, m: int, cutoff: float = 1e-16, jd_tol: float = 1e-8,
                 jd_maxiter: int = 8, device_split: bool = False, alpha=0.0):
        """device_split: split the optimised two-site tensor on the device
        (split_device; needs a DeviceBackend) instead of by host SVDs.
        alpha: the perturbation strength of the state prediction, a number or a function
        of the sweep index (the reference's alpha_initial / alpha_main / alpha_final by
        sweep, ts_optimize.hpp:274-282); nonzero alpha splits by predict_split."""
        self.be, self.model, self.m, self.cutoff = backend, model, m, cutoff
        self.device_split = device_split
        self.alpha = alpha
        self._sweep = 0
        if device_split and (callable(alpha) or alpha != 0.0):
            raise ValueError("the perturbed split runs on the host (dm blocks from the device)")
        self.jd_tol, self.jd_maxiter = jd_tol, jd_maxiter
        self.L = len(tensors)
        self.A = right_canonicalize(tensors)
        self.p12, self.offs = M.fuse_phys(model.phys, model.phys)
        self.W = [M.MPOHandle(w, model.symm) for w in model.mpo]
        self.W12 = [M.MPOHandle(M.twosite_for(model, i), model.symm) for i in range(self.L - 1)]
        # SU2U1: H_eff acts on the spin-reduced two-site tensor (ts_reduction.h; TwoSiteTensor::make_mps,
        # twositetensor.hpp:130-151); the split works on the product-basis tensor
        self.su2 = model.symm == capi.SU2U1
        self.core_energy = getattr(model, "core_energy", 0.0)
        if self.su2 and device_split:
            raise ValueError("the device split takes product-basis two-site tensors; SU2U1 sweeps split on the host")
        self.Lidx = [None] * (self.L + 1)
        self.Lbuf = [None] * (self.L + 1)
        self.Ridx = [None] * (self.L + 1)
        self.Rbuf = [None] * (self.L + 1)
        self.Lidx[0], self.Lbuf[0] = self.be.edge(model.symm, self.A[0].left)
        self.Ridx[self.L], self.Rbuf[self.L] = self.be.edge(model.symm, self.A[-1].right)
        for j in range(self.L - 1, 1, -1):
            self._right_step(j)
        self.log = SweepLog()

    def _left_step(self, j, dev=None):
        self.Lidx[j + 1], self.Lbuf[j + 1] = self.be.left_step(self.model, self.W[j], self.Lidx[j], self.Lbuf[j],
                                                               self.A[j], *(dev or ()))

    def _right_step(self, j, dev=None):
        self.Ridx[j], self.Rbuf[j] = self.be.right_step(self.model, self.W[j], self.Ridx[j + 1], self.Rbuf[j + 1],
                                                        self.A[j], *(dev or ()))

    def optimize_pair(self, i, left_to_right):
        ph = self.log.phase_seconds
        t0 = time.perf_counter()
        psi = twosite(self.A[i], self.A[i + 1], self.p12, self.offs)
        if self.su2:
            from . import su2u1
            psi = su2u1.reduce_twosite(psi, self.model.phys, self.model.phys, self.offs)
        t1 = time.perf_counter()
        extra = {"keep_on_device": True} if self.device_split else {}
        energy, xo, iters, ms = self.be.solve(self.p12, psi, self.W12[i], self.Lidx[i], self.Lbuf[i],
                                              self.Ridx[i + 2], self.Rbuf[i + 2], self.jd_tol, self.jd_maxiter,
                                              **extra)
        t2 = time.perf_counter()
        self.log.hpsi_calls += iters
        self.log.solve_ms += ms
        if self.device_split:
            res = split_device(xo, psi, self.model.phys, self.model.phys, self.offs, self.m, self.cutoff,
                               left_to_right)
        else:
            psi.data = xo
            if self.su2:
                from . import su2u1
                psi = su2u1.unreduce_twosite(psi, self.model.phys, self.model.phys, self.offs)
            alpha = self.alpha(self._sweep) if callable(self.alpha) else self.alpha
            if alpha != 0.0:
                ph_t = time.perf_counter()
                t, _ = theta_site(psi, self.model.phys, self.model.phys, self.offs, left_to_right)
                if left_to_right:
                    dm = self.be.alpha_dm(self.model.phys, self.W[i], self.Lidx[i], self.Lbuf[i], t, alpha, True)
                else:
                    dm = self.be.alpha_dm(self.model.phys, self.W[i + 1], self.Ridx[i + 2], self.Rbuf[i + 2], t,
                                          alpha, False)
                ph["alpha_dm"] = ph.get("alpha_dm", 0.0) + time.perf_counter() - ph_t
                res = predict_split(psi, self.model.phys, self.model.phys, self.offs, self.m, self.cutoff,
                                    left_to_right, dm)
            else:
                res = split(psi, self.model.phys, self.model.phys, self.offs, self.m, self.cutoff, left_to_right)
        self.A[i], self.A[i + 1] = res.A, res.B
        t3 = time.perf_counter()
        if left_to_right:
            self._left_step(i, (res.dev_A, res.dev_A_lp) if res.dev_A is not None else None)
        else:
            self._right_step(i + 1, (res.dev_B,) if res.dev_B is not None else None)
        t4 = time.perf_counter()
        ph["twosite"] = ph.get("twosite", 0.0) + t1 - t0
        ph["site_problem"] = ph.get("site_problem", 0.0) + t2 - t1
        ph["split"] = ph.get("split", 0.0) + t3 - t2
        ph["boundary_step"] = ph.get("boundary_step", 0.0) + t4 - t3
        return energy + self.core_energy, iters, res.truncated_weight

    def sweep(self, sweep_index: int):
        t0 = time.perf_counter()
        self._sweep = sweep_index
        for i in range(0, self.L - 1):
            e, it, tw = self.optimize_pair(i, True)
            self.log.energies.append((sweep_index, i, e, it, tw))
        for i in range(self.L - 2, -1, -1):
            e, it, tw = self.optimize_pair(i, False)
            self.log.energies.append((sweep_index, i, e, it, tw))
        self.be.sync()
        self.log.sweep_seconds.append(time.perf_counter() - t0)
        return self.log.energies[-1][2]
