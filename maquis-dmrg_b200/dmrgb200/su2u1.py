"""Spin-adapted quantum chemistry: the SU2U1 site basis, reduced site operators,
the term list of the reference's qc_su2 model, its MPO and the two-site MPO.

Conventions of the reference (restated, not copied):

* Charges (N, 2S) with fuse = component-wise addition
  (dmrg/framework/dmrg/block_matrix/symmetry/su2u1.h:37-71).  A spatial orbital
  has the four states A = (2,0) doubly occupied, B = (1,1) and C = (1,-1) the
  singly occupied state reached with the total spin going up or down, and
  D = (0,0) empty (models/chem/su2u1/model.hpp:43-62).  B and C are one physical
  spin-1/2 state; the label only records the coupling path, so bond charges
  with 2S < 0 are unphysical and dropped (mps_sectors.h:47-51).
* A reduced site operator is a set of 1x1 blocks (input charge -> output
  charge) with a rank K (twice the spin) and an action, the change of the MPO
  bond spin across the site (SpinDescriptor, block_matrix/symmetry/
  spin_descriptor.h:60-105): a term's bond spins are the running sums of its
  operators' actions.  Blocks B<->C ("full" operators) are present where a
  spin-carrying MPO bond lets the bra and ket coupling paths differ.
* Entry spins (SparseOperator, block_matrix/sparse_operator.h:168-225) are
  |2S| of the state's charge for site operators; for two-site operators they
  are the coupled two-site spins of op_kron (productSpin: C x B is the spin-1
  state, B x C the spin-0 state, spin_descriptor.h:122-134).
* The Hamiltonian is the reference's SU2 term list (models/chem/su2u1/
  model.hpp:345-588, term_maker.h), including its N-conserving rewrite of the
  hopping terms as sum_k c+_i n_k c_j / (N-1); the H_eff it gives is exact in
  the fixed-N sector only.
* The MPO is built from that term list by the bipartite-graph construction of
  qc.build_mpo, with channels labelled by their bond spin, Jordan-Wigner fills
  between fermionic operators and the full identity on spin-1 bonds
  (tagged_mpo_maker_optim.hpp:352-496, insert_filling :535-557).
* The two-site MPO couples the two site operators through the middle bond spin
  into every allowed total rank (make_twosite_mpo / mpo_couple,
  mp_tensors/ts_ops.hpp:40-160; op_kron for SU2,
  block_matrix/site_operator_algorithms.h:204-326).
"""
from __future__ import annotations

import functools
import math
from dataclasses import dataclass

import numpy as np

from . import _capi as capi
from . import mps as S
from .models import Model, MPOTensor, SiteOp, fuse_phys

A, B, C, D = (2, 0), (1, 1), (1, -1), (0, 0)
PHYS = [(A, 1), (B, 1), (C, 1), (D, 1)]

SQ2, SQ3 = math.sqrt(2.0), math.sqrt(3.0)


@dataclass(frozen=True)
class ROp:
    """A reduced site operator: blocks {(in, out): value}, rank K, bond-spin action."""
    name: str
    blocks: tuple
    K: int = 0
    action: int = 0
    fermionic: bool = False


def _rop(name, entries, K=0, action=0, fermionic=False):
    return ROp(name, tuple(sorted(entries.items())), K, action, fermionic)


# site operators of qc_su2 (model.hpp:64-167): (input, output) -> reduced element
_SINGLES = {(B, B): 1.0, (C, C): 1.0}
_FULL = {(B, C): 1.0, (C, B): 1.0}
OPS = {}
for _o in [
    _rop("ident", {(A, A): 1.0, **_SINGLES, (D, D): 1.0}),
    _rop("ident_full", {(A, A): 1.0, **_SINGLES, **_FULL, (D, D): 1.0}),
    _rop("fill", {(A, A): 1.0, (D, D): 1.0, (B, B): -1.0, (C, C): -1.0, (B, C): -1.0, (C, B): -1.0}),
    # creators / destructors: K = 1 (spin 1/2); the action says whether the bond spin goes up or down
    _rop("create_fill", {(B, A): SQ2, (C, A): SQ2, (D, B): 1.0, (D, C): 1.0}, 1, +1, True),
    _rop("create", {(B, A): SQ2, (C, A): SQ2, (D, B): -1.0, (D, C): -1.0}, 1, -1, True),
    _rop("destroy_fill", {(A, B): 1.0, (A, C): 1.0, (B, D): -SQ2, (C, D): -SQ2}, 1, +1, True),
    _rop("destroy", {(A, B): 1.0, (A, C): 1.0, (B, D): SQ2, (C, D): SQ2}, 1, -1, True),
    _rop("create_fill_couple_down", {(B, A): SQ2, (C, A): SQ2, (D, B): 1.0, (D, C): 1.0}, 1, -1, True),
    _rop("destroy_fill_couple_down", {(A, B): 1.0, (A, C): 1.0, (B, D): -SQ2, (C, D): -SQ2}, 1, -1, True),
    _rop("create_couple_up", {(B, A): SQ2, (C, A): SQ2, (D, B): -1.0, (D, C): -1.0}, 1, +1, True),
    _rop("destroy_couple_up", {(A, B): 1.0, (A, C): 1.0, (B, D): SQ2, (C, D): SQ2}, 1, +1, True),
    _rop("create_fill_count", {(B, A): SQ2, (C, A): SQ2}, 1, +1, True),
    _rop("create_count", {(B, A): SQ2, (C, A): SQ2}, 1, -1, True),
    _rop("destroy_fill_count", {(A, B): 1.0, (A, C): 1.0}, 1, +1, True),
    _rop("destroy_count", {(A, B): 1.0, (A, C): 1.0}, 1, -1, True),
    _rop("count", {(A, A): 2.0, **_SINGLES}),
    _rop("count_fill", {(A, A): 2.0, (B, B): -1.0, (C, C): -1.0, (B, C): -1.0, (C, B): -1.0}),
    _rop("docc", {(A, A): 1.0}),
    _rop("e2d", {(D, A): 1.0}),
    _rop("d2e", {(A, D): 1.0}),
    # spin flips: K = 2 (spin 1)
    _rop("flip_to_S2", {(B, B): math.sqrt(1.5), (C, C): math.sqrt(1.5), (B, C): math.sqrt(1.5),
                        (C, B): math.sqrt(1.5)}, 2, +2),
    _rop("flip_to_S0", {(B, B): math.sqrt(1.5), (C, C): math.sqrt(1.5), (B, C): math.sqrt(1.5),
                        (C, B): math.sqrt(1.5)}, 2, -2),
    _rop("flip_S0", {(B, B): math.sqrt(1.5), (C, C): math.sqrt(1.5), (B, C): math.sqrt(1.5),
                     (C, B): math.sqrt(1.5)}, 2, 0),
]:
    OPS[_o.name] = _o

# operator bundles of the term maker (model.hpp:299-343; term_maker.h:38-69)
BUNDLES = {
    "create": dict(couple_up="create_couple_up", couple_down="create", fill_couple_up="create_fill",
                   fill_couple_down="create_fill_couple_down"),
    "destroy": dict(couple_up="destroy_couple_up", couple_down="destroy", fill_couple_up="destroy_fill",
                    fill_couple_down="destroy_fill_couple_down"),
    "create_count": dict(couple_down="create_count", fill_couple_up="create_fill_count"),
    "destroy_count": dict(couple_down="destroy_count", fill_couple_up="destroy_fill_count"),
    "count": dict(no_couple="count", fill_no_couple="count_fill"),
    "flip": dict(no_couple="flip_S0", couple_up="flip_to_S2", couple_down="flip_to_S0"),
}


@functools.lru_cache(maxsize=None)
def site_op(name: str) -> SiteOp:
    """The reduced operator as a SiteOp (1x1 blocks, entry spins |2S| of the charges);
    one shared object per name, so MPO descriptions list each operator once."""
    o = OPS[name]
    blocks = {k: np.array([[v]]) for k, v in o.blocks}
    spins = {k: ([abs(k[0][1])], [abs(k[1][1])]) for k, _ in o.blocks}
    return SiteOp(blocks=blocks, spin=o.K, name=name, spins=spins)


# ---- term list (model.hpp:345-588 with term_maker.h) -----------------------------------------

@dataclass
class Term:
    coeff: float
    ops: list            # [(site, op name)] in any order; sorted by site when the MPO is built
    fermionic: bool = False


def _sgn(*idx) -> bool:
    """Odd permutation parity of the index sequence (term_maker.h:79-90)."""
    inv = sum(1 for a in range(len(idx)) for b in range(a + 1, len(idx)) if idx[a] > idx[b])
    return inv % 2 == 1


def _two_term(sign, scale, i, j, op1, op2):
    return Term(scale, [(i, op1), (j, op2)], sign)


def _positional_two_term(sign, scale, i, j, op1, op1_fill, op2, op2_fill):
    op1_use = op1_fill if i < j else op2_fill
    op2_use = op2 if i < j else op1
    coeff = -scale if (j < i and sign) else scale
    return Term(coeff, [(min(i, j), op1_use), (max(i, j), op2_use)], sign)


def _three_term(scale, pb, p1, p2, boson, boson_fill, op1, op1_fill, op2, op2_fill):
    op1_use = op1_fill if p1 < p2 else op2_fill
    op2_use = op2 if p1 < p2 else op1
    boson_use = boson_fill if (p1 < pb < p2 or p2 < pb < p1) else boson
    coeff = -scale if p2 < p1 else scale
    return Term(coeff, [(pb, boson_use), (min(p1, p2), op1_use), (max(p1, p2), op2_use)], True)


def _four_term(max_two_s, scale, i, j, k, l, op_i, op_k):
    coeff = -scale if _sgn(i, j, k, l) else scale
    st = sorted([(i, op_i), (j, op_i), (k, op_k), (l, op_k)], key=lambda t: t[0])
    bi, bk = BUNDLES[op_i], BUNDLES[op_k]
    pick = lambda t: (bi if t[1] == op_i else bk)
    if max_two_s == 2:
        names = ["fill_couple_up", "couple_up", "fill_couple_down", "couple_down"]
    else:
        names = ["fill_couple_up", "couple_down", "fill_couple_up", "couple_down"]
    return Term(coeff, [(p, pick((p, o))[n]) for (p, o), n in zip(st, names)], True)


_CR, _DE, _CC, _DC = BUNDLES["create"], BUNDLES["destroy"], BUNDLES["create_count"], BUNDLES["destroy_count"]
_CNT, _FL = BUNDLES["count"], BUNDLES["flip"]


def _ssum_two_term(me, i, k, l, j):
    """SpinSumSU2::two_term (term_maker.h:266-278 and two_termA/B1/B2/C)."""
    if i == j and k == l and j != k:
        return [_two_term(False, me, i, k, "count", "count")]
    if i == k and j == l and j != k:
        return [_two_term(False, 2.0 * me, i, j, "e2d", "d2e")]
    if i == l and j == k and i != j:
        return [_positional_two_term(False, SQ3 * me, i, j, _FL["couple_down"], _FL["couple_up"],
                                     _FL["couple_down"], _FL["couple_up"]),
                _two_term(False, -0.5 * me, i, j, "count", "count")]
    if (i == k == l) or (k == l == j) or (i == l == j) or (i == k == j):
        if i == k == l:
            s, p = i, j
        elif k == l == j:
            s, p = j, i
        elif i == l == j:
            s, p = i, k
        else:
            s, p = i, l
        if i == k:
            return [_positional_two_term(True, SQ2 * me, s, p, _CC["couple_down"], _CC["fill_couple_up"],
                                         _DE["couple_down"], _DE["fill_couple_up"])]
        return [_positional_two_term(True, -SQ2 * me, s, p, _DC["couple_down"], _DC["fill_couple_up"],
                                     _CR["couple_down"], _CR["fill_couple_up"])]
    raise ValueError("unexpected index arrangement for a two-index term")


def _ssum_three_term(me, i, k, l, j):
    """SpinSumSU2::three_term (three_termA / three_termB, term_maker.h:280-292, 383-461)."""
    if i == j or k == l:
        if i == j:
            same = i
        if k == l:
            same, k, l = k, i, j
        return [_three_term(SQ2 * me, same, k, l, _CNT["no_couple"], _CNT["fill_no_couple"], _CR["couple_down"],
                            _CR["fill_couple_up"], _DE["couple_down"], _DE["fill_couple_up"])]
    ret = []
    if i == k:
        same, p1, p2 = i, min(l, j), max(l, j)
        ret.append(_three_term(-SQ2 * me, same, p1, p2, "e2d", "e2d", _DE["couple_down"], _DE["fill_couple_up"],
                               _DE["couple_down"], _DE["fill_couple_up"]))
    if j == l:
        same, p1, p2 = j, min(i, k), max(i, k)
        ret.append(_three_term(-SQ2 * me, same, p1, p2, "d2e", "d2e", _CR["couple_down"], _CR["fill_couple_up"],
                               _CR["couple_down"], _CR["fill_couple_up"]))
    if j == k or i == l:
        if j == k:
            same, p1, p2 = j, l, i
        else:
            same, p1, p2 = i, j, k
        phase = -1.0 if _sgn(i, k, l, j) else 1.0
        if same < min(p1, p2):
            ret.append(_three_term(phase * SQ3 * me, same, p1, p2, _FL["couple_up"], _FL["couple_up"],
                                   _CR["couple_down"], _CR["fill_couple_down"], _DE["couple_down"],
                                   _DE["fill_couple_down"]))
            ret.append(_three_term(-0.5 * SQ2 * me, same, p1, p2, "count", "count", _CR["couple_down"],
                                   _CR["fill_couple_up"], _DE["couple_down"], _DE["fill_couple_up"]))
        elif same > max(p1, p2):
            ret.append(_three_term(phase * SQ3 * me, same, p1, p2, _FL["couple_down"], _FL["couple_down"],
                                   _CR["couple_up"], _CR["fill_couple_up"], _DE["couple_up"],
                                   _DE["fill_couple_up"]))
            ret.append(_three_term(-0.5 * SQ2 * me, same, p1, p2, "count", "count", _CR["couple_down"],
                                   _CR["fill_couple_up"], _DE["couple_down"], _DE["fill_couple_up"]))
        else:
            ret.append(_three_term(phase * SQ3 * me, same, p1, p2, _FL["no_couple"], _FL["no_couple"],
                                   _CR["couple_down"], _CR["fill_couple_up"], _DE["couple_down"],
                                   _DE["fill_couple_up"]))
            ret.append(_three_term(-0.5 * SQ2 * me, same, p1, p2, _CNT["fill_no_couple"], _CNT["fill_no_couple"],
                                   _CR["couple_down"], _CR["fill_couple_up"], _DE["couple_down"],
                                   _DE["fill_couple_up"]))
    return ret


def _align(i, j, k, l):
    """chem::align (models/chem/util.h:110-116)."""
    if i < j:
        i, j = j, i
    if k < l:
        k, l = l, k
    if i < k:
        i, k = k, i
        j, l = l, j
    if i == k and j < l:
        j, l = l, j
    return i, j, k, l


def _ssum_four_term(me, i, k, l, j):
    """SpinSumSU2::four_term (term_maker.h:294-329)."""
    i_, j_, k_, l_ = _align(i, j, k, l)
    if k_ > l_ > j_:
        return [_four_term(2, -SQ3 * me, i, k, l, j, "create", "destroy"),
                _four_term(1, me, i, k, l, j, "create", "destroy")]
    if k_ > j_ > l_:
        loc = -me if _sgn(i, k, l, j) else me
        return [_four_term(2, SQ3 * loc, i, k, l, j, "create", "destroy"),
                _four_term(1, loc, i, k, l, j, "create", "destroy")]
    if j_ > k_ > l_:
        return [_four_term(1, 2.0 * me, i, k, l, j, "create", "destroy")]
    raise ValueError("unexpected index arrangement in a four-index term")


def _ssum_v_term(me, i, k, l, j):
    n = len({i, k, l, j})
    if n == 4:
        return _ssum_four_term(me, i, k, l, j)
    if n == 3:
        return _ssum_three_term(me, i, k, l, j)
    if n == 2:
        return _ssum_two_term(me, i, k, l, j)
    return [Term(2.0 * me, [(i, "docc")])]


def integral_elements(h: np.ndarray, eri: np.ndarray, core: float = 0.0, tol: float = 0.0):
    """The unique integrals as the reference reads them (parse_integrals.h:84-156):
    (value, i, j, k, l) with 0-based aligned indices, -1 for an absent index."""
    from .qc import integral_records
    vals, idx = integral_records(h, eri, core, tol)
    out = []
    for v, rec in zip(vals, idx):
        i, j, k, l = (int(x) - 1 for x in rec)
        if (i, j, k, l) != (-1, -1, -1, -1) and abs(v) <= tol:
            continue
        out.append((float(v), *_align(i, j, k, l)))
    return out


def su2_terms(h: np.ndarray, eri: np.ndarray, n_elec: int, core: float = 0.0):
    """(terms, core energy): the reference's qc_su2 create_terms over the unique integrals,
    one- and two-index terms merged by their operator strings (ChemHelperSU2)."""
    L = h.shape[0]
    merged = {}
    core_e = 0.0

    def add(t: Term):
        key = tuple(sorted(t.ops))
        if key in merged:
            merged[key].coeff += t.coeff
        else:
            merged[key] = Term(t.coeff, list(key), t.fermionic)

    for v, i, j, k, l in integral_elements(h, eri, core):
        if (i, j, k, l) == (-1, -1, -1, -1):
            core_e += v
        elif i == j and k == -1 and l == -1:
            add(Term(v, [(i, "count")]))
        elif k == -1 and l == -1:
            if n_elec == 1:
                add(_positional_two_term(True, SQ2 * v, j, i, "create", "create_fill", "destroy", "destroy_fill"))
                add(_positional_two_term(True, SQ2 * v, i, j, "create", "create_fill", "destroy", "destroy_fill"))
            else:
                s = v / (n_elec - 1)
                for kk in range(L):
                    if kk in (i, j):
                        continue
                    for t in _ssum_three_term(s, i, kk, kk, j) + _ssum_three_term(s, j, kk, kk, i):
                        add(t)
                for t in (_ssum_v_term(s, i, i, i, j) + _ssum_v_term(s, j, i, i, i) + _ssum_v_term(s, i, j, j, j)
                          + _ssum_v_term(s, j, j, j, i)):
                    add(t)
        elif i == j == k == l:
            add(Term(v, [(i, "docc")]))
        elif (i == j == k and k != l) or (i != j and j == k == l):
            s_, p_ = (i, l) if i == j else (l, i)
            for t in _ssum_two_term(v, s_, s_, s_, p_) + _ssum_two_term(v, s_, p_, s_, s_):
                add(t)
        elif i == j and k == l and j != k:
            for t in _ssum_two_term(v, i, k, k, i):
                add(t)
        elif i == k and j == l and i != j:
            for t in (_ssum_two_term(0.5 * v, i, i, j, j) + _ssum_two_term(0.5 * v, j, j, i, i)
                      + _ssum_two_term(v, i, j, i, j)):
                add(t)
        elif (i == j and j != k and k != l) or (k == l and i != j and j != k):
            if i == j:
                ts = _ssum_three_term(v, i, k, l, i) + _ssum_three_term(v, i, l, k, i)
            else:
                ts = _ssum_three_term(v, i, k, k, j) + _ssum_three_term(v, j, k, k, i)
            for t in ts:
                add(t)
        elif ((i == k and j != l) or j == k or (j == l and i != k)) and (i != j and k != l):
            for t in (_ssum_three_term(v, i, k, l, j) + _ssum_three_term(v, i, l, k, j)
                      + _ssum_three_term(v, j, k, l, i) + _ssum_three_term(v, j, l, k, i)):
                add(t)
        elif i != j and j != k and k != l and i != k and j != l:
            for t in (_ssum_four_term(v, i, k, l, j) + _ssum_four_term(v, i, l, k, j)
                      + _ssum_four_term(v, j, k, l, i) + _ssum_four_term(v, j, l, k, i)):
                add(t)
        else:
            raise ValueError(f"integral ({i},{j},{k},{l}) matches no term class")
    return [t for t in merged.values() if t.coeff != 0.0], core_e


# ---- MPO ---------------------------------------------------------------------------------------

def _site_sequence(t: Term, L: int):
    """Per-site operator names of a term: its operators at their sites, Jordan-Wigner fills
    where an odd number of fermionic operators follow, the identity elsewhere (the full
    identity on spin-1 bonds), None outside the term's span; and its bond spins."""
    ops = sorted(t.ops)
    seq = [None] * L
    spins = [0] * (L + 1)
    sites = [p for p, _ in ops]
    if len(set(sites)) != len(sites):
        raise ValueError("two operators of one term on one site")
    nferm_after = [sum(OPS[o].fermionic for _, o in ops[a + 1:]) for a in range(len(ops))]
    spin = 0
    for a, (p, name) in enumerate(ops):
        seq[p] = name
        spin += OPS[name].action
        nxt = ops[a + 1][0] if a + 1 < len(ops) else p + 1
        for q in range(p + 1, nxt):
            seq[q] = "fill" if nferm_after[a] % 2 else ("ident_full" if spin > 1 else "ident")
    if spin != 0:
        raise ValueError("term does not couple to total spin 0")
    return seq


def _min_vertex_cover(nu: int, nv: int, adj: list):
    from .qc import _min_vertex_cover as mvc
    return mvc(nu, nv, adj)


def build_mpo(terms: list, L: int) -> list:
    """Site MPO tensors (models.MPOTensor with bond spins) of sum_terms coeff * ops by the
    bipartite-graph construction; the operators at each (b1, b2) are kept by name with
    their summed coefficients (several ranks may meet there)."""
    acc = {}
    for t in terms:
        key = tuple(_site_sequence(t, L))
        acc[key] = acc.get(key, 0.0) + t.coeff
    cur = {(0, key): c for key, c in acc.items() if c != 0.0}
    spin_of = {0: 0}
    mpo, nprev = [], 1
    for s in range(L):
        uidx, vidx, edges = {}, {}, {}
        for (chan, rest), c in cur.items():
            u = uidx.setdefault((chan, rest[0] or "ident"), len(uidx))
            v = vidx.setdefault(rest[1:], len(vidx))
            edges[(u, v)] = edges.get((u, v), 0.0) + c
        ulist = list(uidx)
        W = {}

        def put(b1, b2, name, c):
            d = W.setdefault((b1, b2), {})
            d[name] = d.get(name, 0.0) + c

        nxt, new_spin = {}, {}
        if s == L - 1:
            for (u, v), c in edges.items():
                chan, op = ulist[u]
                put(chan, 0, op, c)
            ncol = 1
            new_spin = {0: 0}
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
                put(chan, n, op, 1.0)
                new_spin[n] = spin_of[chan] + OPS[op].action
            for (u, v), c in edges.items():
                if u in new_u:
                    key = (new_u[u], vlist[v])
                    nxt[key] = nxt.get(key, 0.0) + c
                else:
                    chan, op = ulist[u]
                    n = new_v[v]
                    put(chan, n, op, c)
                    sp_ = spin_of[chan] + OPS[op].action
                    if new_spin.setdefault(n, sp_) != sp_:
                        raise ValueError("inconsistent bond spins in the MPO construction")
                    nxt[(n, vlist[v])] = 1.0
            ncol = len(new_u) + len(new_v)
        tensor_terms = {}
        for (b1, b2), d in W.items():
            lst = [(site_op(name), c) for name, c in sorted(d.items()) if c != 0.0]
            if lst:
                tensor_terms[(b1, b2)] = lst
        lspin = [spin_of[b] for b in range(nprev)]
        rspin = [new_spin[b] for b in range(ncol)]
        mpo.append(MPOTensor(nprev, ncol, tensor_terms, left_spin=lspin, right_spin=rspin))
        cur, nprev, spin_of = nxt, ncol, new_spin
    return mpo


# ---- two-site MPO (ts_ops.hpp:40-160, op_kron SU2 site_operator_algorithms.h:204-326) -----------

def _product_spin(a, b) -> int:
    if a[1] == -1 and b[1] == 1:
        return 2
    return abs(a[1] + b[1])


def allowed_spins(left: int, right: int, k1: int, k2: int):
    """Ranks k of the product of ranks k1, k2 that can couple bond spins left -> right."""
    return [k for k in range(abs(k1 - k2), k1 + k2 + 1, 2) if abs(k - left) <= right <= k + left]


def _op_entries(op: SiteOp):
    return {k: float(v[0, 0]) for k, v in op.blocks.items()}


def op_kron(op1: SiteOp, op2: SiteOp, j: int, jpp: int, jp: int, k: int, p12_offs):
    """Two-site reduced operator of rank k from op1 (site 1) and op2 (site 2) with left,
    middle and right bond spins j, jpp, jp.  Blocks {(in, out): {(r, c): value}} and
    entry spins {(in, out): ({r: J}, {c: J'})}."""
    a, b = _op_entries(op1), _op_entries(op2)
    k1, k2 = op1.spin, op2.spin
    # a rank-0 partner of a rank > 0 operator acts on both coupling paths of the singly
    # occupied state (the reference expands its identity the same way)
    if k1 > 0 and k2 == 0 and (B, C) not in b:
        b[(B, C)] = 1.0
        b[(C, B)] = 1.0
    if k1 == 0 and k2 > 0 and (B, C) not in a:
        a[(B, C)] = 1.0
        a[(C, B)] = 1.0
    glob = math.sqrt((jpp + 1) * (k + 1)) * capi.lib.dmrgb200_wigner6j(j, jp, k, k2, k1, jpp)
    if ((j + jp + k1 + k2) // 2) % 2:
        glob = -glob
    blocks, spins = {}, {}
    for (ia, oa), va in a.items():
        for (ib, ob), vb in b.items():
            nl = (ia[0] + ib[0], ia[1] + ib[1])
            nr = (oa[0] + ob[0], oa[1] + ob[1])
            r, c = p12_offs[(ia, ib)], p12_offs[(oa, ob)]
            J, Jp = _product_spin(ia, ib), _product_spin(oa, ob)
            cpl = mod_coupling(abs(ia[1]), abs(ib[1]), J, k1, k2, k, abs(oa[1]), abs(ob[1]), Jp)
            blk = blocks.setdefault((nl, nr), {})
            blk[(r, c)] = blk.get((r, c), 0.0) + va * vb * cpl * glob
            rs, cs = spins.setdefault((nl, nr), ({}, {}))
            rs[r] = J
            cs[c] = Jp
    return blocks, spins


def mod_coupling(a, b, c, d, e, f, g, h, i) -> float:
    return math.sqrt((g + 1) * (h + 1) * (c + 1) * (f + 1)) * capi.lib.dmrgb200_wigner9j(a, b, c, d, e, f, g, h, i)


def twosite_mpo(W1: MPOTensor, W2: MPOTensor, phys1=PHYS, phys2=PHYS, tol: float = 1e-15) -> MPOTensor:
    """W12(b1, b3) = sum over b2 and over the allowed total ranks k of the coupled products
    of W1(b1, b2) and W2(b2, b3), one two-site operator per (b1, b3, k) with scale 1."""
    p12, offs = fuse_phys(phys1, phys2)
    dims = dict(p12)
    out1, out2 = {}, {}
    for (b1, b2) in W1.terms:
        out1.setdefault(b1, []).append(b2)
    for (b2, b3) in W2.terms:
        out2.setdefault(b2, []).append(b3)
    paths = {}
    for b1 in sorted(out1):
        for b2 in sorted(out1[b1]):
            for b3 in out2.get(b2, ()):
                paths.setdefault((b1, b3), []).append(b2)
    terms = {}
    cache = {}  # the coupled product depends only on the two operators and the three bond spins

    def kron(o1, o2, j, jpp, jp, k):
        key = (o1.name, o2.name, j, jpp, jp, k)
        if key not in cache:
            cache[key] = op_kron(o1, o2, j, jpp, jp, k, offs)
        return cache[key]

    for (b1, b3) in sorted(paths):
        j, jp = W1.left_spin[b1], W2.right_spin[b3]
        coupled = {}
        for b2 in sorted(paths[(b1, b3)]):
            jpp = W1.right_spin[b2]
            for o1, s1 in W1.terms[(b1, b2)]:
                for o2, s2 in W2.terms[(b2, b3)]:
                    for k in allowed_spins(j, jp, o1.spin, o2.spin):
                        blocks, spins = kron(o1, o2, j, jpp, jp, k)
                        acc_b, acc_s = coupled.setdefault(k, ({}, {}))
                        for key, ent in blocks.items():
                            d = acc_b.setdefault(key, {})
                            for rc, v in ent.items():
                                d[rc] = d.get(rc, 0.0) + v * s1 * s2
                            rs, cs = acc_s.setdefault(key, ({}, {}))
                            rs.update(spins[key][0])
                            cs.update(spins[key][1])
        lst = []
        for k in sorted(coupled):
            acc_b, acc_s = coupled[k]
            blocks, bspins = {}, {}
            for key, ent in acc_b.items():
                if not any(abs(v) > tol for v in ent.values()):
                    continue
                nl, nr = key
                M = np.zeros((dims[nl], dims[nr]))
                for (r, c), v in ent.items():
                    if abs(v) > tol:
                        M[r, c] = v
                blocks[key] = M
                rs, cs = acc_s[key]
                bspins[key] = ([rs.get(r, 0) for r in range(dims[nl])], [cs.get(c, 0) for c in range(dims[nr])])
            if blocks:
                lst.append((SiteOp(blocks=blocks, spin=k, name=f"ts{k}", spins=bspins), 1.0))
        if lst:
            terms[(b1, b3)] = lst
    return MPOTensor(W1.row_dim, W2.col_dim, terms, left_spin=list(W1.left_spin), right_spin=list(W2.right_spin))


# ---- model ---------------------------------------------------------------------------------------

def allowed_sectors(L: int, total, Mmax: int, phys=PHYS):
    """Bond sectors of an L-orbital SU2U1 chain ending in `total` = (N, 2S): every
    product charge with 2S >= 0 reachable from both ends, multiplicities (numbers of
    coupling paths, i.e. of spin multiplets) capped at Mmax (mps_sectors.h:53-140)."""
    def prod(ph, idx):
        out = {}
        for pc, d in ph:
            for c, m in idx:
                f = (pc[0] + c[0], pc[1] + c[1])
                if f[1] < 0:
                    continue
                out[f] = out.get(f, 0) + d * m
        return sorted(out.items())
    left = [[((0, 0), 1)]]
    for _ in range(L):
        left.append(prod(phys, left[-1]))
    neg = [((-c[0], -c[1]), d) for c, d in phys]
    right = [None] * (L + 1)
    right[L] = [(tuple(total), 1)]
    for i in range(L - 1, -1, -1):
        right[i] = prod(neg, right[i + 1])
    out = []
    for i in range(L + 1):
        rd = dict(right[i])
        out.append(sorted((c, min(Mmax, m, rd[c])) for c, m in left[i] if c in rd))
    return out


def synthetic_bonds(L: int, total, m: int, radius: float = 3.5):
    """Synthetic SU2U1 bond sectors of total multiplet count about m: the weights of
    mps.synthetic_sectors over the physical (N, 2S) charges, with the mean charge
    (N i / L, 2S i / L)."""
    allowed = allowed_sectors(L, total, 10 ** 9)
    return [S.synthetic_sectors(PHYS, L, tuple(total), m, i, radius, allowed) for i in range(L + 1)]


def quantum_chemistry(L: int, n_elec: int, two_s: int = 0, h=None, eri=None, core: float = 0.0,
                      seed_h: int = 3, seed_b: int = 4) -> Model:
    """SU2U1 quantum-chemistry model on L orbitals with n_elec electrons and total spin
    two_s / 2; the integrals default to qc.synthetic_integrals(L).  `core_energy` is the
    constant the reference adds to the reported energy (ts_optimize.hpp:269-272)."""
    from . import qc
    if h is None or eri is None:
        h, eri = qc.synthetic_integrals(L, seed_h, seed_b)
    terms, core_e = su2_terms(h, eri, n_elec, core)
    mpo = build_mpo(terms, L)
    m = Model("quantum_chemistry_su2u1", capi.SU2U1, PHYS, {}, mpo, (n_elec, two_s), [])
    m.h, m.eri, m.core_energy, m.su2_terms = h, eri, core_e, terms
    return m


# ---- spin-reduced two-site tensor (ts_reduction.h:36-333) --------------------------------------

def _coupling_6j(jl: int, jr: int, j: int, s1: int, s2: int, jm: int) -> float:
    c = math.sqrt((j + 1) * (jm + 1)) * capi.lib.dmrgb200_wigner6j(jl, jr, j, s2, s1, jm)
    return -c if ((jl + jr + s1 + s2) // 2) % 2 else c


def _recouple(psi: S.SiteTensor, phys1, phys2, offs, reduce: bool) -> S.SiteTensor:
    """reduce=True: the product-basis two-site tensor (one slot per pair of site states,
    the middle spin of the pair given by the first state's label) -> the spin-reduced
    two-site tensor (the pair coupled to total spin 0 or 1 in the B x C / C x B slots)
    (ts_reduction::reduce_right); reduce=False: the inverse (unreduce_right)."""
    out = S.SiteTensor(psi.phys, psi.left, psi.right)
    for (lb, s, ss), (_, c0, ml, mr, rb) in psi.rp.sub.items():
        lc = psi.left[lb][0]
        rc = psi.right[rb][0]
        sc = psi.phys[s][0]
        jl, jr = lc[1], rc[1]
        # the site pair (c1, c2) of this slot
        pair = None
        for c1, _ in phys1:
            for c2, _ in phys2:
                if (c1[0] + c2[0], c1[1] + c2[1]) == sc and offs[(c1, c2)] == ss:
                    pair = (c1, c2)
        if pair is None:
            continue
        c1, c2 = pair
        s1, s2 = abs(c1[1]), abs(c2[1])
        src = S.block_view(psi.data, psi.rp, lb)[:, c0:c0 + mr]
        if jl == jr and jl > 0 and s1 == 1 and s2 == 1:
            if reduce:
                jm = jl + c1[1]
                base = ss if c1[1] == 1 else ss - 1
                for j in (0, 2):
                    c = _coupling_6j(jl, jr, j, s1, s2, jm)
                    _, d0, _, _, _ = out.rp.sub[(lb, s, base + j // 2)]
                    S.block_view(out.data, out.rp, lb)[:, d0:d0 + mr] += c * src
            else:
                j = 0 if c1[1] == 1 else 2
                base = ss if j == 0 else ss - 1
                for jm in (jl - 1, jl + 1):
                    c = _coupling_6j(jl, jr, j, s1, s2, jm)
                    _, d0, _, _, _ = out.rp.sub[(lb, s, base + 1 if jm == jl - 1 else base)]
                    S.block_view(out.data, out.rp, lb)[:, d0:d0 + mr] += c * src
        else:
            j = abs(c1[1] + c2[1])
            jm = jl + c1[1]
            if jm < 0:
                continue
            c = _coupling_6j(jl, jr, j, s1, s2, jm)
            S.block_view(out.data, out.rp, lb)[:, c0:c0 + mr] += c * src
    return out


def reduce_twosite(psi: S.SiteTensor, phys1=PHYS, phys2=PHYS, offs=None) -> S.SiteTensor:
    if offs is None:
        offs = fuse_phys(phys1, phys2)[1]
    return _recouple(psi, phys1, phys2, offs, True)


def unreduce_twosite(psi: S.SiteTensor, phys1=PHYS, phys2=PHYS, offs=None) -> S.SiteTensor:
    if offs is None:
        offs = fuse_phys(phys1, phys2)[1]
    return _recouple(psi, phys1, phys2, offs, False)
