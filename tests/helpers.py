"""Shared test fixtures: small chains with boundaries built by the CPU oracle."""
import numpy as np

from dmrgb200 import engine as E
from dmrgb200 import models as M
from dmrgb200 import mps as S

import oracle as O


def unit_mask(t: S.SiteTensor) -> np.ndarray:
    m = np.zeros(t.rp.total, dtype=bool)
    for b in range(len(t.rp.rows)):
        m[t.rp.offs[b]:t.rp.offs[b] + t.rp.rows[b] * t.rp.cols[b]] = True
    return m


def random_psi(p12, left, right, rng) -> S.SiteTensor:
    psi = S.SiteTensor(p12, left, right)
    psi.data[unit_mask(psi)] = rng.standard_normal(int(unit_mask(psi).sum()))
    return psi


class OracleChain:
    """Boundaries L (bond i) and R (bond i+2) from oracle boundary steps and the
    two-site H·psi schedule at sites (i, i+1)."""

    def __init__(self, model, bonds, tensors, i, symmetric=True):
        self.model, self.bonds, self.tensors, self.i = model, bonds, tensors, i
        L = len(tensors)
        Lidx = E.edge_bindex(model.symm, bonds[0])
        Lval = Lidx.edge_values()
        for p in range(i):
            W = M.MPOHandle(model.mpo[p], model.symm)
            sch, nidx = E.schedule_left_step(model.phys, bonds[p], bonds[p + 1], W, Lidx, symmetric)
            Lval = O.left_step(sch.plan, Lval, Lidx, tensors[p].data, tensors[p].left_paired(), nidx)
            Lidx = nidx
        Ridx = E.edge_bindex(model.symm, bonds[L])
        Rval = Ridx.edge_values()
        for p in range(L - 1, i + 1, -1):
            W = M.MPOHandle(model.mpo[p], model.symm)
            sch, nidx = E.schedule_right_step(model.phys, bonds[p], bonds[p + 1], W, Ridx, symmetric)
            Rval = O.right_step(sch.plan, Rval, Ridx, tensors[p].data, tensors[p].data, nidx)
            Ridx = nidx
        self.Lidx, self.Lval, self.Ridx, self.Rval = Lidx, Lval, Ridx, Rval
        self.p12, _ = M.fuse_phys(model.phys, model.phys)
        self.W12 = M.MPOHandle(M.twosite_mpo(model.mpo[i], model.mpo[i + 1], model.phys, model.phys), model.symm)
        self.left, self.right = bonds[i], bonds[i + 2]
        self.sched = E.schedule_hpsi(self.p12, self.left, self.right, self.W12, Lidx, Ridx)

    def hpsi(self, x):
        return O.hpsi(self.sched.plan, self.Lval, self.Lidx, self.Rval, self.Ridx, x)


def make_chain(name, L, Mmax, seed=0, synthetic_m=None):
    model = {"heisenberg": lambda: M.heisenberg(L),
             "hubbard": lambda: M.fermi_hubbard(L),
             "bose": lambda: M.bose_hubbard(L, N=L // 2)}[name]()
    rng = np.random.default_rng(seed)
    if synthetic_m is None:
        bonds = S.allowed_sectors(model.phys, L, model.total_charge, Mmax)
    else:
        bonds = [S.synthetic_sectors(model.phys, L, model.total_charge, synthetic_m, i) for i in range(L + 1)]
    tensors = S.random_mps(model.phys, bonds, rng)
    return model, bonds, tensors, rng
