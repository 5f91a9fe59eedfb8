"""Block-sparse MPS site tensors and their FP64 memory layouts.

Layouts (all blocks column-major, each block padded to 128 elements like the
reference's DavidsonVector, dmrg/framework/dmrg/solver/davidson_vector.cpp:87-152):
  right-paired: one block per left sector lc, rows m_l(lc), columns ordered by
                physical sector s (index order) then copy ss, each m_r(lc + s)
                wide (out_right_pb, site_hamil_schedule.hpp:61-63);
  left-paired:  one block per right sector rc, rows ordered by s then ss, each
                m_l(rc - s) high, columns m_r(rc) (move_boundary.hpp:186).
"""
from __future__ import annotations

import math

import numpy as np

PAD = 128


def cadd(a, b):
    return (a[0] + b[0], a[1] + b[1])


def csub(a, b):
    return (a[0] - b[0], a[1] - b[1])


def round_up(v, a=PAD):
    return (v + a - 1) // a * a


class Layout:
    def __init__(self, rows, cols, offs, total, sub):
        self.rows, self.cols, self.offs, self.total = rows, cols, offs, total
        self.sub = sub  # (block, s, ss) -> (row0, col0, nrows, ncols) of that sub-block


def right_paired_layout(phys, left, right):
    rpos = {c: i for i, (c, _) in enumerate(right)}
    rows, cols, offs, sub, total = [], [], [], {}, 0
    for lb, (lc, ml) in enumerate(left):
        c = 0
        for s, (sc, d) in enumerate(phys):
            rc = cadd(lc, sc)
            if rc not in rpos:
                continue
            mr = right[rpos[rc]][1]
            for ss in range(d):
                sub[(lb, s, ss)] = (0, c + ss * mr, ml, mr, rpos[rc])
            c += d * mr
        rows.append(ml)
        cols.append(c)
        offs.append(total)
        total += round_up(ml * c)
    return Layout(rows, cols, offs, total, sub)


def left_paired_layout(phys, left, right):
    lpos = {c: i for i, (c, _) in enumerate(left)}
    rows, cols, offs, sub, total = [], [], [], {}, 0
    for rb, (rc, mr) in enumerate(right):
        r = 0
        for s, (sc, d) in enumerate(phys):
            lc = csub(rc, sc)
            if lc not in lpos:
                continue
            ml = left[lpos[lc]][1]
            for ss in range(d):
                sub[(rb, s, ss)] = (r + ss * ml, 0, ml, mr, lpos[lc])
            r += d * ml
        rows.append(r)
        cols.append(mr)
        offs.append(total)
        total += round_up(r * mr)
    return Layout(rows, cols, offs, total, sub)


def block_view(flat, lay, b):
    n = lay.rows[b] * lay.cols[b]
    return flat[lay.offs[b]:lay.offs[b] + n].reshape(lay.cols[b], lay.rows[b]).T  # column-major view


class SiteTensor:
    """MPS site tensor stored right-paired (flat FP64 vector)."""

    def __init__(self, phys, left, right, data=None):
        self.phys, self.left, self.right = list(phys), list(left), list(right)
        self.rp = right_paired_layout(self.phys, self.left, self.right)
        self.data = np.zeros(self.rp.total) if data is None else np.asarray(data, dtype=np.float64)
        assert self.data.shape == (self.rp.total,)

    def left_paired(self) -> np.ndarray:
        lp = left_paired_layout(self.phys, self.left, self.right)
        out = np.zeros(lp.total)
        lpos = {c: i for i, (c, _) in enumerate(self.left)}
        for (rb, s, ss), (r0, _, ml, mr, lb) in lp.sub.items():
            _, c0, _, _, _ = self.rp.sub[(lb, s, ss)]
            src = block_view(self.data, self.rp, lb)[:, c0:c0 + mr]
            block_view(out, lp, rb)[r0:r0 + ml, :] = src
        del lpos
        return out

    def norm(self) -> float:
        return float(np.linalg.norm(self.data))

    def dense(self) -> np.ndarray:
        """Dense [D_left, d, D_right] array over the full bond and physical bases."""
        loff = np.cumsum([0] + [m for _, m in self.left])
        roff = np.cumsum([0] + [m for _, m in self.right])
        poff = np.cumsum([0] + [d for _, d in self.phys])
        A = np.zeros((loff[-1], poff[-1], roff[-1]))
        for (lb, s, ss), (_, c0, ml, mr, rb) in self.rp.sub.items():
            A[loff[lb]:loff[lb] + ml, poff[s] + ss, roff[rb]:roff[rb] + mr] = \
                block_view(self.data, self.rp, lb)[:, c0:c0 + mr]
        return A


def index_product(phys, idx, cap=None):
    """Charges of phys x idx with summed multiplicities (Index operator*), capped."""
    out = {}
    order = []
    for pc, d in phys:
        for c, m in idx:
            f = cadd(pc, c)
            if f not in out:
                out[f] = 0
                order.append(f)
            out[f] += d * m
    if cap is not None:
        for f in out:
            out[f] = min(cap, out[f])
    return [(f, out[f]) for f in order]


def allowed_sectors(phys, L, total, Mmax):
    """Bond sectors of an L-site chain ending in `total` with every sector capped at
    Mmax (allowed_sectors, dmrg/framework/dmrg/mp_tensors/mps_sectors.h:53-140)."""
    ident = (0, 0)
    left = [[(ident, 1)]]
    for i in range(1, L + 1):
        left.append(index_product(phys, left[-1], Mmax))
    neg = [((-c[0], -c[1]), d) for c, d in phys]
    right = [None] * (L + 1)
    right[L] = [(total, 1)]
    for i in range(L - 1, -1, -1):
        right[i] = index_product(neg, right[i + 1], Mmax)
    out = []
    for i in range(L + 1):
        rd = dict(right[i])
        sec = [(c, min(Mmax, m, rd[c])) for c, m in left[i] if c in rd]
        out.append(sorted(sec))
    return out


def synthetic_bonds(phys, L, total, m, radius=3.5):
    """synthetic_sectors for every bond 0..L."""
    allowed = allowed_sectors(phys, L, total, 10 ** 9)
    return [synthetic_sectors(phys, L, total, m, i, radius, allowed) for i in range(L + 1)]


def synthetic_sectors(phys, L, total, m, i, radius=3.5, allowed_all=None):
    """Bond-i sectors of a synthetic state of total bond dimension about m.

    Converged DMRG states concentrate their Schmidt spectrum on charges near the
    mean charge of the left block, with the number of kept states falling off
    roughly quadratically in the charge deviation.  Here every allowed charge q
    of bond i gets the weight max(0, 1 - |q - q_mean|^2 / radius^2), with
    q_mean = total * i / L (radius in units of the charge lattice); each sector
    receives a share of m proportional to its weight, at least 1, capped by the
    exact multiplicity bound of allowed_sectors, and sectors whose share is
    below 0.5 are dropped."""
    if allowed_all is None:
        allowed_all = allowed_sectors(phys, L, total, 10 ** 9)
    allowed = dict(allowed_all[i])
    if i == 0 or i == L:
        return sorted(allowed.items())
    qm = (total[0] * i / L, total[1] * i / L)
    wts = {c: max(0.0, 1.0 - ((c[0] - qm[0]) ** 2 + (c[1] - qm[1]) ** 2) / radius ** 2) for c in allowed}
    tot = sum(wts.values())
    if tot == 0:
        best = min(allowed, key=lambda c: (c[0] - qm[0]) ** 2 + (c[1] - qm[1]) ** 2)
        return [(best, int(min(allowed[best], m)))]
    out = []
    for c in sorted(allowed):
        share = m * wts[c] / tot
        if share < 0.5:
            continue
        out.append((c, int(min(allowed[c], max(1, round(share))))))
    return out


def random_mps(phys, bonds, rng: np.random.Generator, normalize=True):
    """Site tensors with uniform[0,1) entries on every allowed block, each
    normalised (mpstensor.hpp:71-72, mps_initializers.h:68-71)."""
    mps = []
    for i in range(len(bonds) - 1):
        t = SiteTensor(phys, bonds[i], bonds[i + 1])
        for (lb, s, ss), (_, c0, ml, mr, rb) in t.rp.sub.items():
            block_view(t.data, t.rp, lb)[:, c0:c0 + mr] = rng.random((ml, mr))
        if normalize:
            n = t.norm()
            if n > 0:
                t.data /= n
        mps.append(t)
    return mps
