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


def spin_sector_spectrum_jw(h: np.ndarray, eri: np.ndarray, n_elec: int, two_s: int) -> np.ndarray:
    """Exact (FCI) eigenvalues of the ab-initio Hamiltonian with integrals (h, eri) in the
    sector of n_elec electrons and total spin two_s / 2, ascending: H in the spin-orbital
    basis (TwoU1 model, Sz = S), restricted to the eigenspace S^2 = S(S+1) of the dense
    S^2 = sum_ab (S+_a S-_b + S-_a S+_b) / 2 + Sz_a Sz_b.  The reference for SU2U1 results
    (whose H_eff acts on spin multiplets)."""
    from dmrgb200 import qc
    L = h.shape[0]
    nu, nd = (n_elec + two_s) // 2, (n_elec - two_s) // 2
    m = qc.quantum_chemistry(L, nu, nd, h=h, eri=eri)
    mask = sector_mask(m, L, (nu, nd))
    H = sparse_hamiltonian(m, L)[mask][:, mask].toarray()
    loc = dict(m.local)
    splus = loc["cdag_up"] @ loc["c_down"]
    loc.update(splus=splus, sminus=splus.T.copy(), sz=np.diag([0.0, 0.5, -0.5, 0.0]))
    spin_terms = []
    for a in range(L):
        for b in range(L):
            spin_terms += [(0.5, [(a, "splus"), (b, "sminus")]), (0.5, [(a, "sminus"), (b, "splus")]),
                           (1.0, [(a, "sz"), (b, "sz")])]
    ms = M.Model("spin_squared", m.symm, m.phys, loc, [], m.total_charge, spin_terms, fermionic_ops=m.fermionic_ops)
    S2 = sparse_hamiltonian(ms, L)[mask][:, mask].toarray()
    w, V = np.linalg.eigh(S2)
    s = two_s / 2
    Q = V[:, np.abs(w - s * (s + 1)) < 1e-8]
    return np.sort(np.linalg.eigvalsh(Q.T @ H @ Q))


def _strings(L: int, n: int):
    from itertools import combinations
    return [sum(1 << p for p in c) for c in combinations(range(L), n)]


def _excitation(strings, L):
    """e[p][q]: sparse matrix of a+_p a_q on one spin's occupation strings (sign from the
    occupied orbitals between p and q)."""
    pos = {s: k for k, s in enumerate(strings)}
    n = len(strings)
    out = [[None] * L for _ in range(L)]
    for p in range(L):
        for q in range(L):
            rows, cols, vals = [], [], []
            for k, st in enumerate(strings):
                if not (st >> q) & 1:
                    continue
                t = st & ~(1 << q)
                if (t >> p) & 1:
                    continue
                sign = (-1) ** bin(st & ((1 << q) - 1)).count("1") * (-1) ** bin(t & ((1 << p) - 1)).count("1")
                rows.append(pos[t | (1 << p)])
                cols.append(k)
                vals.append(sign)
            out[p][q] = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    return out


def spin_sector_spectrum(h: np.ndarray, eri: np.ndarray, n_elec: int, two_s: int) -> np.ndarray:
    """Exact (FCI) eigenvalues of H = sum h_pq E_pq + 1/2 sum (pq|rs) (E_pq E_rs - d_qr E_ps)
    (E_pq = sum over spin of a+_p a_q) on the spin multiplets of n_elec electrons and total
    spin two_s / 2, ascending.  The determinants of the sector Sz = S are alpha x beta
    occupation strings; the states with total spin S are those annihilated by
    S+ = sum_p a+_(p alpha) a_(p beta) (the highest-weight states of each multiplet)."""
    L = h.shape[0]
    nu, nd = (n_elec + two_s) // 2, (n_elec - two_s) // 2
    sa, sb = _strings(L, nu), _strings(L, nd)
    ea, eb = _excitation(sa, L), _excitation(sb, L)
    Ia, Ib = sp.identity(len(sa), format="csr"), sp.identity(len(sb), format="csr")
    E = [[sp.kron(ea[p][q], Ib, format="csr") + sp.kron(Ia, eb[p][q], format="csr") for q in range(L)]
         for p in range(L)]
    H = sp.csr_matrix((len(sa) * len(sb),) * 2)
    for p in range(L):
        for q in range(L):
            F = sp.csr_matrix(H.shape)
            for r in range(L):
                for s_ in range(L):
                    if eri[p, q, r, s_] != 0.0:
                        F = F + eri[p, q, r, s_] * E[r][s_]
            H = H + h[p, q] * E[p][q] + 0.5 * (E[p][q] @ F)
            for s_ in range(L):
                H = H - 0.5 * eri[p, q, q, s_] * E[p][s_]
    H = H.toarray()
    if two_s < nd + nu:
        # S+ from (nu, nd) to (nu + 1, nd - 1): a+_(p alpha) a_(p beta), alpha orbitals ordered first
        if nd == 0:
            Q = np.eye(H.shape[0])
        else:
            ta, tb = _strings(L, nu + 1), _strings(L, nd - 1)
            pa, pb = {x: k for k, x in enumerate(ta)}, {x: k for k, x in enumerate(tb)}
            rows, cols, vals = [], [], []
            for ia, a in enumerate(sa):
                for ib, b in enumerate(sb):
                    for p in range(L):
                        if not (b >> p) & 1 or (a >> p) & 1:
                            continue
                        b2, a2 = b & ~(1 << p), a | (1 << p)
                        sign = (-1) ** (nu + bin(b & ((1 << p) - 1)).count("1")) * \
                            (-1) ** bin(a & ((1 << p) - 1)).count("1")
                        rows.append(pa[a2] * len(tb) + pb[b2])
                        cols.append(ia * len(sb) + ib)
                        vals.append(sign)
            Sp = sp.csr_matrix((vals, (rows, cols)), shape=(len(ta) * len(tb), H.shape[0])).toarray()
            _, sv, Vt = np.linalg.svd(Sp)
            rank = int(np.sum(sv > 1e-10))
            Q = Vt[rank:].T
    else:
        Q = np.eye(H.shape[0])
    return np.sort(np.linalg.eigvalsh(Q.T @ H @ Q))
