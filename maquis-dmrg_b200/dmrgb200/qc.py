"""Quantum-chemistry Hamiltonian in spatial orbitals with TwoU1 symmetry.

    H = sum_{ij,s} h_ij c+_is c_js + 1/2 sum_{ijkl,s,t} (ij|kl) c+_is c+_kt c_lt c_js

(the reference's quantum_chemistry model, models/chem/, in the spin-orbital
TwoU1 form; one site per spatial orbital with the basis |0>, |up>, |down>,
|up down> of the coded Fermi-Hubbard model).  The MPO is built from the term
list by the bipartite-graph construction (Ren, Li, Jiang, Shuai, J. Chem. Phys.
153, 084118 (2020)): at every bond the terms split into a left part (the MPO
channel they came from and the operator on the new site) and a right part (the
operators still to come); a minimum vertex cover of that bipartite graph (Konig's
theorem from a maximum matching) gives the channels of the next bond, which keeps
the bond dimension near its minimum without any SVD.  Jordan-Wigner strings are
folded into the site operators: after the operators of a term are sorted by site
(with the sign of the permutation), the operator on site q is the product of the
term's operators on q followed by the fill operator F when an odd number of the
term's fermionic operators sit to the right of q.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import maximum_bipartite_matching

from . import _capi as capi
from .models import Model, MPOTensor, op_from_dense

_E, _A, _B, _D = (0, 0), (1, 0), (0, 1), (1, 1)   # |0>, |up>, |down>, |up down> = c+_up c+_down |0>
PHYS = [(_E, 1), (_A, 1), (_B, 1), (_D, 1)]


def local_ops() -> dict:
    """Dense local operators O[out, in] in the basis of PHYS (as in models.fermi_hubbard)."""
    cu_dag = np.zeros((4, 4))
    cu_dag[1, 0] = 1.0
    cu_dag[3, 2] = 1.0
    cd_dag = np.zeros((4, 4))
    cd_dag[2, 0] = 1.0
    cd_dag[3, 1] = -1.0
    return dict(ident=np.eye(4), fill=np.diag([1.0, -1.0, -1.0, 1.0]), cdag_up=cu_dag, c_up=cu_dag.T.copy(),
                cdag_down=cd_dag, c_down=cd_dag.T.copy())


def synthetic_integrals(L: int, seed_h: int = 3, seed_b: int = 4, n_aux: int | None = None):
    """Seeded synthetic integrals: h symmetric with off-diagonal N(0, 0.5^2) and a
    diagonal uniform in [-2, -0.5] sorted ascending; (ij|kl) = sum_P B^P_ij B^P_kl
    with symmetric B^P of N(0, 0.1^2) entries, P = 1 .. n_aux (default 2 L), which
    makes the ERIs 8-fold symmetric and positive semi-definite."""
    rng = np.random.default_rng(seed_h)
    h = rng.normal(0.0, 0.5, (L, L))
    h = np.triu(h, 1)
    h = h + h.T
    h[np.diag_indices(L)] = np.sort(rng.uniform(-2.0, -0.5, L))
    rngb = np.random.default_rng(seed_b)
    n_aux = 2 * L if n_aux is None else n_aux
    B = rngb.normal(0.0, 0.1, (n_aux, L, L))
    B = 0.5 * (B + B.transpose(0, 2, 1))
    eri = np.einsum("pij,pkl->ijkl", B, B)
    return h, eri


FERMIONIC = ("cdag_up", "c_up", "cdag_down", "c_down")


def qc_terms(h: np.ndarray, eri: np.ndarray, tol: float = 0.0) -> list:
    """[(coeff, [(site, op), ...])] in operator order (the dense builder's format)."""
    L = h.shape[0]
    terms = []
    spins = ("up", "down")
    for i in range(L):
        for j in range(L):
            if abs(h[i, j]) > tol:
                for s in spins:
                    terms.append((h[i, j], [(i, "cdag_" + s), (j, "c_" + s)]))
    for i in range(L):
        for j in range(L):
            for k in range(L):
                for l in range(L):
                    v = 0.5 * eri[i, j, k, l]
                    if abs(v) <= tol:
                        continue
                    for s in spins:
                        for t in spins:
                            if (i == k and s == t) or (j == l and s == t):
                                continue  # c+ c+ or c c on one spin orbital
                            terms.append((v, [(i, "cdag_" + s), (k, "cdag_" + t), (l, "c_" + t), (j, "c_" + s)]))
    return terms


def site_ordered(ops: list, L: int, local: dict):
    """(sign, [matrix or None per site]) of a product of operators given in
    operator order: sorted by site with the sign of the fermionic permutation, the
    Jordan-Wigner fill folded into the site operators (None = identity)."""
    seq = list(ops)
    sign = 1
    # stable insertion sort by site; swapping two fermionic operators flips the sign
    for a in range(1, len(seq)):
        b = a
        while b > 0 and seq[b - 1][0] > seq[b][0]:
            if seq[b - 1][1] in FERMIONIC and seq[b][1] in FERMIONIC:
                sign = -sign
            seq[b - 1], seq[b] = seq[b], seq[b - 1]
            b -= 1
    out = [None] * L
    nferm = [0] * (L + 1)  # fermionic operators on sites >= q
    for site, name in seq:
        if name in FERMIONIC:
            nferm[site] += 1
    for q in range(L - 1, -1, -1):
        nferm[q] += nferm[q + 1]
    lo = min(site for site, _ in seq)
    hi = max(site for site, _ in seq)
    for q in range(lo, hi + 1):
        m = None
        for site, name in seq:
            if site == q:
                m = local[name] if m is None else m @ local[name]
        if (nferm[q + 1] % 2) == 1:
            m = local["fill"] if m is None else m @ local["fill"]
        out[q] = m
    return sign, out


def _min_vertex_cover(nu: int, nv: int, adj: list):
    """Minimum vertex cover (cover_u, cover_v) of a bipartite graph from a maximum
    matching (Konig's theorem): alternating search from the unmatched left vertices."""
    rows = [u for u in range(nu) for _ in adj[u]]
    cols = [v for u in range(nu) for v in adj[u]]
    g = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(nu, nv))
    match_u = maximum_bipartite_matching(g, perm_type="column")
    match_v = np.full(nv, -1)
    for u, v in enumerate(match_u):
        if v >= 0:
            match_v[v] = u
    seen_u = np.zeros(nu, dtype=bool)
    seen_v = np.zeros(nv, dtype=bool)
    stack = [u for u in range(nu) if match_u[u] < 0]
    seen_u[stack] = True
    while stack:
        u = stack.pop()
        for v in adj[u]:
            if seen_v[v] or match_u[u] == v:
                continue
            seen_v[v] = True
            u2 = match_v[v]
            if u2 >= 0 and not seen_u[u2]:
                seen_u[u2] = True
                stack.append(u2)
    return ~seen_u, seen_v


def build_mpo(terms: list, L: int, local: dict, phys) -> list:
    """Site MPO tensors of sum_terms coeff * prod ops (bipartite-graph construction)."""
    registry, mats = {}, [np.eye(4)]

    def reg(m):
        if m is None:
            return 0
        key = (m + 0.0).tobytes()
        if key not in registry:
            registry[key] = len(mats)
            mats.append(m)
        return registry[key]

    acc = {}
    for coeff, ops in terms:
        sign, ms = site_ordered(ops, L, local)
        if any(m is not None and not np.any(m) for m in ms):
            continue
        key = tuple(reg(m) for m in ms)
        acc[key] = acc.get(key, 0.0) + sign * coeff
    cur = {(0, key): c for key, c in acc.items() if c != 0.0}
    mpo, nprev = [], 1
    for s in range(L):
        uidx, vidx, edges = {}, {}, {}
        for (chan, rest), c in cur.items():
            u = uidx.setdefault((chan, rest[0]), len(uidx))
            v = vidx.setdefault(rest[1:], len(vidx))
            edges[(u, v)] = edges.get((u, v), 0.0) + c
        ulist = list(uidx)
        W = {}

        def put(b1, b2, m):
            W[(b1, b2)] = W.get((b1, b2), 0) + m

        nxt = {}
        if s == L - 1:
            for (u, v), c in edges.items():
                chan, op = ulist[u]
                put(chan, 0, c * mats[op])
            ncol = 1
        else:
            adj = [[] for _ in ulist]
            for (u, v) in edges:
                adj[u].append(v)
            cover_u, cover_v = _min_vertex_cover(len(ulist), len(vidx), adj)
            vlist = list(vidx)
            new_u = {u: i for i, u in enumerate(np.nonzero(cover_u)[0])}
            new_v = {v: len(new_u) + i for i, v in enumerate(np.nonzero(cover_v)[0])}
            for u, n in new_u.items():
                chan, op = ulist[u]
                put(chan, n, mats[op])
            for (u, v), c in edges.items():
                if u in new_u:
                    key = (new_u[u], vlist[v])
                    nxt[key] = nxt.get(key, 0.0) + c
                else:
                    chan, op = ulist[u]
                    n = new_v[v]
                    put(chan, n, c * mats[op])
                    nxt[(n, vlist[v])] = 1.0
            ncol = len(new_u) + len(new_v)
        tensor_terms = {}
        for (b1, b2), m in W.items():
            if np.any(m):
                tensor_terms[(b1, b2)] = [(op_from_dense(m, phys), 1.0)]
        mpo.append(MPOTensor(nprev, ncol, tensor_terms))
        cur, nprev = nxt, ncol
    return mpo


def quantum_chemistry(L: int, n_up: int, n_down: int, h=None, eri=None, seed_h: int = 3, seed_b: int = 4) -> Model:
    """QC model on L spatial orbitals with n_up / n_down electrons (TwoU1)."""
    if h is None or eri is None:
        h, eri = synthetic_integrals(L, seed_h, seed_b)
    local = local_ops()
    terms = qc_terms(h, eri)
    mpo = build_mpo(terms, L, local, PHYS)
    m = Model("quantum_chemistry", capi.TWOU1, PHYS, local, mpo, (n_up, n_down), terms, fermionic_ops=FERMIONIC)
    m.h, m.eri = h, eri
    return m


# ---- integral derivatives ------------------------------------------------------------
#
# The MPO coefficients (and so the plan's term alphas) are linear in every
# integral, and the bipartite construction's structure does not depend on the
# integrals' values, so d(alpha)/d(integral) is the change of the alphas when the
# integral is raised by one.  An integral stands for its symmetry orbit:
# h_ab = h_ba, and (ab|cd) with its 8-fold symmetry.

def integral_orbit(which: str, index) -> set:
    """Index tuples that share the value of integral `which` ("h" or "eri") at `index`."""
    if which == "h":
        a, b = index
        return {(a, b), (b, a)}
    a, b, c, d = index
    return {(a, b, c, d), (b, a, c, d), (a, b, d, c), (b, a, d, c),
            (c, d, a, b), (d, c, a, b), (c, d, b, a), (d, c, b, a)}


def raise_integral(h: np.ndarray, eri: np.ndarray, which: str, index, delta: float):
    """Copies of (h, eri) with the integral's orbit raised by delta."""
    h, eri = h.copy(), eri.copy()
    for idx in integral_orbit(which, index):
        if which == "h":
            h[idx] += delta
        else:
            eri[idx] += delta
    return h, eri


def integral_operator_terms(which: str, index) -> list:
    """dH/d(integral) as a term list [(coeff, [(site, op), ...])] (format of qc_terms)."""
    terms = []
    spins = ("up", "down")
    for idx in integral_orbit(which, index):
        if which == "h":
            p, q = idx
            for s in spins:
                terms.append((1.0, [(p, "cdag_" + s), (q, "c_" + s)]))
        else:
            p, q, r, t = idx
            for s in spins:
                for u in spins:
                    if (p == r and s == u) or (q == t and s == u):
                        continue
                    terms.append((0.5, [(p, "cdag_" + s), (r, "cdag_" + u), (t, "c_" + u), (q, "c_" + s)]))
    return terms


def operator_model(model: Model, terms: list) -> Model:
    """The model's sites and symmetry with the MPO of another term list (an
    observable such as dH/d(integral)), for expectation values through the same
    boundary steps and H·psi."""
    L = len(model.mpo)
    mpo = build_mpo(terms, L, model.local, model.phys)
    return Model(model.name + "_operator", model.symm, model.phys, model.local, mpo, model.total_charge, terms,
                 fermionic_ops=model.fermionic_ops)


# ---- integral files -------------------------------------------------------------------
#
# The reference's integral text format (models/chem/parse_integrals.h:36-62, 134-146):
# four header lines, then records "value i j k l" with 1-based orbital indices,
# 0 for an absent index: (ij|kl) as "v i j k l", h_ij as "v i j 0 0", the core
# energy as "v 0 0 0 0".  Only one representative of each symmetry orbit is listed.
# The binary form (the `integrals` parameter, parse_integrals.h:64-80) is all
# values as doubles followed by all indices as 32-bit ints, four per record.

def integral_records(h: np.ndarray, eri: np.ndarray, core: float = 0.0, tol: float = 0.0):
    """(values, indices[n, 4]) of the unique entries: (ij|kl) with i >= j, k >= l and
    (i, j) >= (k, l) (pairs compared as i*(i+1)/2 + j), h_ij with i >= j, then the core
    energy; 1-based indices, entries with |value| <= tol skipped (the core always kept)."""
    L = h.shape[0]
    vals, idx = [], []
    for i in range(L):
        for j in range(i + 1):
            ij = i * (i + 1) // 2 + j
            for k in range(L):
                for l in range(k + 1):
                    if k * (k + 1) // 2 + l > ij:
                        continue
                    v = float(eri[i, j, k, l])
                    if abs(v) > tol:
                        vals.append(v)
                        idx.append((i + 1, j + 1, k + 1, l + 1))
    for i in range(L):
        for j in range(i + 1):
            v = float(h[i, j])
            if abs(v) > tol:
                vals.append(v)
                idx.append((i + 1, j + 1, 0, 0))
    vals.append(float(core))
    idx.append((0, 0, 0, 0))
    return np.array(vals), np.array(idx, dtype=np.int32).reshape(-1, 4)


def write_integrals(path, h: np.ndarray, eri: np.ndarray, core: float = 0.0, tol: float = 0.0,
                    header=("synthetic integrals", "", "", "")) -> int:
    """Write the text format (values to 17 significant digits, so they read back
    exactly); returns the number of records."""
    vals, idx = integral_records(h, eri, core, tol)
    with open(path, "w") as f:
        for line in list(header)[:4] + [""] * (4 - len(header)):
            f.write(line + "\n")
        for v, (i, j, k, l) in zip(vals, idx):
            f.write(f"{v:.17g} {i} {j} {k} {l}\n")
    return len(vals)


def integrals_buffer(h: np.ndarray, eri: np.ndarray, core: float = 0.0, tol: float = 0.0) -> bytes:
    """The binary form: all values (float64), then all indices (int32, four per record)."""
    vals, idx = integral_records(h, eri, core, tol)
    return vals.astype("<f8").tobytes() + idx.astype("<i4").tobytes()


def _expand(vals, idx, L: int, order=None, cutoff: float = 0.0):
    """h, eri (8-fold symmetric) and the core energy from records; `order` (1-based,
    the orbital at each site, as the reference's orbital_order) maps orbitals to sites."""
    if order is None:
        site = np.arange(L)
    else:
        order = np.asarray(order) - 1
        if sorted(order.tolist()) != list(range(L)):
            raise ValueError("orbital_order must be a permutation of 1..L")
        site = np.empty(L, dtype=int)
        site[order] = np.arange(L)
    h = np.zeros((L, L))
    eri = np.zeros((L, L, L, L))
    core = 0.0
    for v, rec in zip(vals, idx):
        if abs(v) <= cutoff and tuple(rec) != (0, 0, 0, 0):
            continue
        i, j, k, l = (int(x) for x in rec)
        if (i, j, k, l) == (0, 0, 0, 0):
            core += v
        elif k == 0 and l == 0:
            a, b = site[i - 1], site[j - 1]
            h[a, b] = h[b, a] = v
        else:
            a, b, c, d = site[i - 1], site[j - 1], site[k - 1], site[l - 1]
            for p in integral_orbit("eri", (a, b, c, d)):
                eri[p] = v
    return h, eri, core


def read_integrals(path, L: int, order=None, cutoff: float = 0.0):
    """Parse the text format: skip four header lines, read records of five numbers."""
    with open(path) as f:
        for _ in range(4):
            f.readline()
        raw = np.array(f.read().split(), dtype=np.float64)
    if raw.size % 5:
        raise ValueError("integral parsing failed: the record count is not a multiple of 5")
    rec = raw.reshape(-1, 5)
    return _expand(rec[:, 0], rec[:, 1:].astype(int), L, order, cutoff)


def parse_integrals_buffer(buf: bytes, L: int, order=None, cutoff: float = 0.0):
    """Parse the binary form."""
    line = 8 + 4 * 4
    if len(buf) % line:
        raise ValueError("integral buffer parsing failed: size is not a multiple of one record")
    n = len(buf) // line
    vals = np.frombuffer(buf[:8 * n], dtype="<f8")
    idx = np.frombuffer(buf[8 * n:], dtype="<i4").reshape(n, 4)
    return _expand(vals, idx, L, order, cutoff)
