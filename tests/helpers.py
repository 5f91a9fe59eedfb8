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

    def __init__(self, model, bonds, tensors, i, symmetric=True, merge=True):
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
        self.W12mpo = M.twosite_for(model, i, merge=merge)
        self.W12 = M.MPOHandle(self.W12mpo, model.symm)
        self.left, self.right = bonds[i], bonds[i + 2]
        self.sched = E.schedule_hpsi(self.p12, self.left, self.right, self.W12, Lidx, Ridx)

    def hpsi(self, x):
        return O.hpsi(self.sched.plan, self.Lval, self.Lidx, self.Rval, self.Ridx, x)


def make_chain(name, L, Mmax, seed=0, synthetic_m=None):
    from dmrgb200 import qc
    model = {"heisenberg": lambda: M.heisenberg(L),
             "hubbard": lambda: M.fermi_hubbard(L),
             "bose": lambda: M.bose_hubbard(L, N=L // 2),
             "qc": lambda: qc.quantum_chemistry(L, L // 2, L // 2)}[name]()
    rng = np.random.default_rng(seed)
    if synthetic_m is None:
        bonds = S.allowed_sectors(model.phys, L, model.total_charge, Mmax)
    else:
        bonds = [S.synthetic_sectors(model.phys, L, model.total_charge, synthetic_m, i) for i in range(L + 1)]
    tensors = S.random_mps(model.phys, bonds, rng)
    return model, bonds, tensors, rng


# ---- adjoint fixtures ---------------------------------------------------------------

def perturbed_mpo(W: M.MPOTensor, key, delta: float) -> M.MPOTensor:
    """Copy of W with the scale of term key = (b1, b2, j) shifted by delta."""
    import copy
    terms = {k: list(v) for k, v in W.terms.items()}
    b1, b2, j = key
    op, sc = terms[(b1, b2)][j]
    terms[(b1, b2)][j] = (op, sc + delta)
    Wp = copy.copy(W)
    Wp.terms = terms
    return Wp


def hubbard_center_terms(handle: M.MPOHandle, W12: M.MPOTensor):
    """Two-site (unmerged) term indices of the Fermi-Hubbard FSM MPO whose scale is
    proportional to the hopping across the centre bond (0 -> {1..4} -> 5), to U of
    the first site (0 -> 5 -> 5) and to U of the second site (0 -> 0 -> 5)."""
    out = {"t": [], "U1": [], "U2": []}
    for idx, (b1, b3, j) in enumerate(handle.term_keys):
        (_, b2, _), _ = W12.sources[(b1, b3)][j]
        if (b1, b3) != (0, 5):
            continue
        if b2 in (1, 2, 3, 4):
            out["t"].append(idx)
        elif b2 == 5:
            out["U1"].append(idx)
        elif b2 == 0:
            out["U2"].append(idx)
    return out


def hubbard_derivative_ops(model, i: int):
    """dH/dt of the hopping across bond (i, i+1) and dH/dU of sites i and i+1, as
    term lists of the model's dense builder."""
    hop = []
    for s in ("up", "down"):
        hop.append((-1.0, [(i, "cdag_" + s), (i + 1, "c_" + s)]))
        hop.append((-1.0, [(i + 1, "cdag_" + s), (i, "c_" + s)]))
    return {"t": hop, "U1": [(1.0, [(i, "docc")])], "U2": [(1.0, [(i + 1, "docc")])]}


# ---- quantum-chemistry derivative fixtures ---------------------------------------------

def qc_integral_derivative(model, L, i, ch, galpha, which, index):
    """d<w|H_eff x>/d(integral) from the per-term derivatives galpha: the plan is
    rebuilt with the integral raised by one (alpha is linear in every integral and
    the MPO structure does not depend on its value) over the same boundaries.
    which = "h" (index (a, b), symmetric pair) or "eri" (index (a, b, c, d), its
    8-fold orbit).  Returns (derivative, dense term list of dH/d(integral))."""
    from dmrgb200 import qc
    h, eri = qc.raise_integral(model.h, model.eri, which, index, 1.0)
    terms = qc.integral_operator_terms(which, index)
    m2 = qc.quantum_chemistry(L, model.total_charge[0], model.total_charge[1], h=h, eri=eri)
    W12 = M.MPOHandle(M.twosite_mpo(m2.mpo[i], m2.mpo[i + 1], m2.phys, m2.phys), m2.symm)
    s = E.schedule_hpsi(ch.p12, ch.left, ch.right, W12, ch.Lidx, ch.Ridx)
    base = ch.sched.plan
    for key in ("term_t", "term_col", "l_term", "l_b1"):
        assert np.array_equal(base[key], s.plan[key]), "MPO structure changed with the integral"
    return float(np.asarray(galpha) @ (s.plan["term_alpha"] - base["term_alpha"])), terms
