"""ORACLE — test infrastructure only.  Dense exact references for small chains.

* dense Hamiltonians built directly from each model's term list (fermionic
  operators with explicit Jordan-Wigner strings), independent of the MPO code;
* exact ground states by diagonalisation in a fixed charge sector;
* the dense embedding P of a two-site tensor into the full Hilbert space, so that
  H_eff = P^T H P is the matrix the schedule-based H·psi must apply.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from dmrgb200 import models as M
from dmrgb200 import mps as S


def local_charges(model: M.Model):
    return [c for c, d in model.phys for _ in range(d)]


def sparse_hamiltonian(model: M.Model, L: int):
    """H from the model's term list (sparse CSR), fermionic operators carrying
    explicit Jordan-Wigner strings on the sites to their left."""
    d = sum(dd for _, dd in model.phys)
    F = sp.csr_matrix(model.local["fill"]) if "fill" in model.local else None
    I = sp.identity(d, format="csr")

    def site_op(name, p):
        O = sp.csr_matrix(model.local[name])
        out = None
        for q in range(L):
            mq = O if q == p else (F if (q < p and name in model.fermionic_ops) else I)
            out = mq if out is None else sp.kron(out, mq, format="csr")
        return out

    H = sp.csr_matrix((d ** L, d ** L))
    for coeff, factors in model.dense_terms:
        term = None
        for p, name in factors:
            o = site_op(name, p)
            term = o if term is None else term @ o
        H = H + coeff * term
    return H.tocsr()


def dense_hamiltonian(model: M.Model, L: int) -> np.ndarray:
    return sparse_hamiltonian(model, L).toarray()


def sector_mask(model: M.Model, L: int, total) -> np.ndarray:
    ch = np.array(local_charges(model))
    d = len(ch)
    q = np.zeros((d ** L, 2), dtype=int)
    idx = np.arange(d ** L)
    for p in range(L - 1, -1, -1):
        q += ch[idx % d]
        idx //= d
    return (q[:, 0] == total[0]) & (q[:, 1] == total[1])


def ground_energy(model: M.Model, L: int) -> float:
    H = sparse_hamiltonian(model, L)
    idx = np.nonzero(sector_mask(model, L, model.total_charge))[0]
    Hs = H[idx][:, idx]
    if Hs.shape[0] <= 2000:
        return float(np.linalg.eigvalsh(Hs.toarray())[0])
    return float(spl.eigsh(Hs, k=1, which="SA", tol=1e-13, maxiter=100000)[0][0])


def mps_dense(tensors) -> np.ndarray:
    """Contract site tensors (dense [Dl, d, Dr]) into a vector (site 0 most significant)."""
    v = tensors[0]
    for t in tensors[1:]:
        v = np.tensordot(v, t, axes=([v.ndim - 1], [0]))
    return v.reshape(-1)


def twosite_dense(phys1, phys2, psi: S.SiteTensor) -> np.ndarray:
    """Dense [Dl, d1, d2, Dr] of a two-site tensor whose physical index is the
    fused basis of models.fuse_phys(phys1, phys2)."""
    A = psi.dense()  # [Dl, d12, Dr] in fused-basis order
    p12, offs = M.fuse_phys(phys1, phys2)
    poff12 = {}
    o = 0
    for c, d in p12:
        poff12[c] = o
        o += d
    d1s, d2s = dict(phys1), dict(phys2)
    o1 = np.cumsum([0] + [d for _, d in phys1])
    o2 = np.cumsum([0] + [d for _, d in phys2])
    out = np.zeros((A.shape[0], o1[-1], o2[-1], A.shape[2]))
    for a, (c1, _) in enumerate(phys1):
        for b, (c2, _) in enumerate(phys2):
            f = (c1[0] + c2[0], c1[1] + c2[1])
            for i1 in range(d1s[c1]):
                for i2 in range(d2s[c2]):
                    k = poff12[f] + offs[(c1, c2)] + i1 * d2s[c2] + i2
                    out[:, o1[a] + i1, o2[b] + i2, :] = A[:, k, :]
    return out


def embedding(mps_left, mps_right, phys1, phys2, left, right, p12) -> np.ndarray:
    """Columns: dense states of every unit two-site tensor (P of H_eff = P^T H P)."""
    tmpl = S.SiteTensor(p12, left, right)
    n = tmpl.rp.total
    cols = []
    lefts = [t.dense() for t in mps_left]
    rights = [t.dense() for t in mps_right]
    valid = np.zeros(n, dtype=bool)
    for b in range(len(tmpl.rp.rows)):
        valid[tmpl.rp.offs[b]:tmpl.rp.offs[b] + tmpl.rp.rows[b] * tmpl.rp.cols[b]] = True
    P = []
    for k in range(n):
        if not valid[k]:
            P.append(None)
            continue
        e = np.zeros(n)
        e[k] = 1.0
        psi = S.SiteTensor(p12, left, right, e)
        core = twosite_dense(phys1, phys2, psi)
        D = core.shape
        core = core.reshape(D[0], D[1] * D[2], D[3])
        P.append(mps_dense(lefts + [core] + rights))
    dim = len(next(p for p in P if p is not None))
    return np.stack([p if p is not None else np.zeros(dim) for p in P], axis=1)


def mpo_dense(model: M.Model, L: int) -> np.ndarray:
    """Dense H from the site MPOs: contract W_0 ... W_{L-1} over the bond indices."""
    d = sum(dd for _, dd in model.phys)
    offs = {}
    o = 0
    for c, dd in model.phys:
        offs[c] = o
        o += dd

    def dense_op(op):
        O = np.zeros((d, d))
        for (cin, cout), B in op.blocks.items():
            for i in range(B.shape[0]):
                for j in range(B.shape[1]):
                    O[offs[cout] + j, offs[cin] + i] += B[i, j]
        return O

    # env[b] = operator on sites < p ending in bond state b
    env = {0: np.eye(1)}
    for p in range(L):
        W = model.mpo[p]
        new = {}
        for (b1, b2), terms in W.terms.items():
            if b1 not in env:
                continue
            O = sum(sc * dense_op(op) for op, sc in terms)
            new[b2] = new.get(b2, 0) + np.kron(env[b1], O)
        env = new
    return env[0]
