"""Lattice models, their site operators and MPOs (inputs of the hot path).

Operator convention (the reference's SiteOperator / SparseOperator,
dmrg/framework/dmrg/block_matrix/sparse_operator.h:35-235): an operator is a
set of blocks keyed by (input charge, output charge); block entry (i, j) is
<out j| O |in i>.  Here every operator is built from a dense local matrix
O[out, in] over the physical basis and split into charge blocks.

Models (coded models of the reference):
  heisenberg       U1, charges 2Sz = +-1          (models/coded/models_u1.hpp:38-166)
  fermi_hubbard    TwoU1, charges (N_up, N_down)  (models/coded/models_2u1.hpp:39-)
  bose_hubbard     U1, charges N = 0..Nmax        (models/coded/models_u1.hpp:296-490)
Each MPO is a nearest-neighbour finite-state machine whose bond indices carry
Hermitian partners (the reference's MPOTensor_detail::Hermitian), so symmetric
boundary steps can skip the conjugate blocks.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi

Charge = tuple  # (q0, q1)


@dataclass
class SiteOp:
    blocks: dict  # (cin, cout) -> np.ndarray (d_in x d_out), entry <out|O|in>
    spin: int = 0
    name: str = ""
    spins: dict = None  # SU2 only: (cin, cout) -> (row spins, column spins) of the block's entries


@dataclass
class MPOTensor:
    row_dim: int
    col_dim: int
    terms: dict  # (b1, b2) -> list[(SiteOp, scale)]
    left_herm: list = None   # partner per left bond index or None
    left_phase: list = None
    right_herm: list = None
    right_phase: list = None
    left_spin: list = None
    right_spin: list = None
    sources: dict = None     # (b1, b2) -> per-term provenance (twosite_mpo(merge=False))


@dataclass
class Model:
    name: str
    symm: int
    phys: list          # [(charge, dim)]
    local: dict         # name -> dense local O[out, in]
    mpo: list           # [MPOTensor] per site
    total_charge: Charge
    dense_terms: list = field(default_factory=list)  # [(coeff, [(site, opname), ...])] for exact diagonalisation
    fermionic_ops: tuple = ()


def phys_states(phys):
    """Flat list of (charge, sub-index) in basis order."""
    out = []
    for c, d in phys:
        for k in range(d):
            out.append((c, k))
    return out


def op_from_dense(O: np.ndarray, phys, name="") -> SiteOp:
    """Split a dense local operator O[out, in] into charge blocks (in, out)."""
    st = phys_states(phys)
    offs, o = {}, 0
    for c, d in phys:
        offs[c] = o
        o += d
    dims = dict(phys)
    blocks = {}
    for cin, din in phys:
        for cout, dout in phys:
            B = np.zeros((din, dout))
            for i in range(din):
                for j in range(dout):
                    B[i, j] = O[offs[cout] + j, offs[cin] + i]
            if np.any(B != 0):
                blocks[(cin, cout)] = B
    del st, dims
    return SiteOp(blocks=blocks, name=name)


def _fsm_mpo(L: int, D: int, bulk: dict, first_row: int, last_col: int, herm: dict, phases: dict) -> list:
    """Site MPOs from a bulk finite-state machine: bulk[(b1, b2)] = [(op, scale)].

    Site 0 keeps only row `first_row`; site L-1 keeps only column `last_col`.
    `herm`/`phases` give Hermitian partners of the bulk bond indices."""
    mpo = []
    for p in range(L):
        rows = [first_row] if p == 0 else list(range(D))
        cols = [last_col] if p == L - 1 else list(range(D))
        rmap = {b: i for i, b in enumerate(rows)}
        cmap = {b: i for i, b in enumerate(cols)}
        terms = {}
        for (b1, b2), lst in bulk.items():
            if b1 in rmap and b2 in cmap:
                terms[(rmap[b1], cmap[b2])] = list(lst)

        def hp(idx):
            partner, ph = [], []
            for b in idx:
                q = herm.get(b)
                partner.append(None if q is None or q not in idx else idx.index(q))
                ph.append(phases.get(b, 1))
            return partner, ph

        lh, lp = hp(rows)
        rh, rp = hp(cols)
        mpo.append(MPOTensor(len(rows), len(cols), terms, lh, lp, rh, rp))
    return mpo


def heisenberg(L: int, Jxy: float = 1.0, Jz: float = 1.0, sz_total: int = 0) -> Model:
    up, dn = (1, 0), (-1, 0)
    phys = [(up, 1), (dn, 1)]
    I = np.eye(2)
    Sp = np.array([[0.0, 1.0], [0.0, 0.0]])   # basis order (up, down): S+ |dn> = |up>
    Sm = Sp.T.copy()
    Sz = np.diag([0.5, -0.5])
    ops = {k: op_from_dense(v, phys, k) for k, v in dict(ident=I, splus=Sp, sminus=Sm, sz=Sz).items()}
    # 0: nothing placed, 1: S+ placed, 2: S- placed, 3: Sz placed, 4: complete
    bulk = {(0, 0): [(ops["ident"], 1.0)], (0, 1): [(ops["splus"], Jxy / 2)], (0, 2): [(ops["sminus"], Jxy / 2)],
            (0, 3): [(ops["sz"], Jz)], (1, 4): [(ops["sminus"], 1.0)], (2, 4): [(ops["splus"], 1.0)],
            (3, 4): [(ops["sz"], 1.0)], (4, 4): [(ops["ident"], 1.0)]}
    herm = {0: 0, 1: 2, 2: 1, 3: 3, 4: 4}
    mpo = _fsm_mpo(L, 5, bulk, 0, 4, herm, {})
    dense = []
    for p in range(L - 1):
        dense += [(Jz, [(p, "sz"), (p + 1, "sz")]), (Jxy / 2, [(p, "splus"), (p + 1, "sminus")]),
                  (Jxy / 2, [(p, "sminus"), (p + 1, "splus")])]
    return Model("heisenberg", capi.U1, phys, dict(ident=I, splus=Sp, sminus=Sm, sz=Sz), mpo, (sz_total, 0), dense)


def fermi_hubbard(L: int, t: float = 1.0, U: float = 4.0, n_up: int | None = None, n_down: int | None = None) -> Model:
    e, a, b, d = (0, 0), (1, 0), (0, 1), (1, 1)   # |0>, |up>, |down>, |up down> = c+_up c+_down |0>
    phys = [(e, 1), (a, 1), (b, 1), (d, 1)]
    cu_dag = np.zeros((4, 4))
    cu_dag[1, 0] = 1.0   # |0> -> |up>
    cu_dag[3, 2] = 1.0   # |down> -> |up down>
    cd_dag = np.zeros((4, 4))
    cd_dag[2, 0] = 1.0   # |0> -> |down>
    cd_dag[3, 1] = -1.0  # |up> -> c+_down c+_up |0> = -|up down>
    cu, cd = cu_dag.T.copy(), cd_dag.T.copy()
    F = np.diag([1.0, -1.0, -1.0, 1.0])
    I = np.eye(4)
    D = np.diag([0.0, 0.0, 0.0, 1.0])
    local = dict(ident=I, fill=F, cdag_up=cu_dag, c_up=cu, cdag_down=cd_dag, c_down=cd, docc=D,
                 cdag_up_F=cu_dag @ F, c_up_F=cu @ F, cdag_down_F=cd_dag @ F, c_down_F=cd @ F)
    ops = {k: op_from_dense(v, phys, k) for k, v in local.items()}
    # c+_i c_j (j = i+1) = [c+ F]_i [c]_j ;  c+_j c_i = -[c F]_i [c+]_j
    # 0: nothing placed, 1..4: hop pending, 5: complete
    bulk = {(0, 0): [(ops["ident"], 1.0)],
            (0, 1): [(ops["cdag_up_F"], -t)], (0, 2): [(ops["c_up_F"], t)],
            (0, 3): [(ops["cdag_down_F"], -t)], (0, 4): [(ops["c_down_F"], t)],
            (0, 5): [(ops["docc"], U)],
            (1, 5): [(ops["c_up"], 1.0)], (2, 5): [(ops["cdag_up"], 1.0)],
            (3, 5): [(ops["c_down"], 1.0)], (4, 5): [(ops["cdag_down"], 1.0)],
            (5, 5): [(ops["ident"], 1.0)]}
    herm = {0: 0, 1: 2, 2: 1, 3: 4, 4: 3, 5: 5}
    mpo = _fsm_mpo(L, 6, bulk, 0, 5, herm, {})
    n_up = L // 2 if n_up is None else n_up
    n_down = L // 2 if n_down is None else n_down
    dense = []
    for p in range(L):
        dense.append((U, [(p, "docc")]))
    for p in range(L - 1):
        for s in ("up", "down"):
            dense.append((-t, [(p, "cdag_" + s), (p + 1, "c_" + s)]))
            dense.append((-t, [(p + 1, "cdag_" + s), (p, "c_" + s)]))
    return Model("fermi_hubbard", capi.TWOU1, phys, local, mpo, (n_up, n_down), dense,
                 fermionic_ops=("cdag_up", "c_up", "cdag_down", "c_down"))


def bose_hubbard(L: int, t: float = 1.0, U: float = 8.0, V: float = 0.0, Nmax: int = 2, N: int | None = None) -> Model:
    phys = [((n, 0), 1) for n in range(Nmax + 1)]
    dim = Nmax + 1
    bdag = np.zeros((dim, dim))
    for n in range(1, Nmax + 1):
        bdag[n, n - 1] = np.sqrt(n)
    bb = bdag.T.copy()
    nop = np.diag(np.arange(dim, dtype=float))
    inter = np.diag([n * n - n for n in range(dim)]).astype(float)
    I = np.eye(dim)
    local = dict(ident=I, create=bdag, destroy=bb, count=nop, interaction=inter)
    ops = {k: op_from_dense(v, phys, k) for k, v in local.items()}
    # 0: nothing placed, 1: b+ placed, 2: b placed, 3: n placed, 4: complete
    bulk = {(0, 0): [(ops["ident"], 1.0)], (0, 1): [(ops["create"], -t)], (0, 2): [(ops["destroy"], -t)],
            (0, 4): [(ops["interaction"], U / 2)], (1, 4): [(ops["destroy"], 1.0)], (2, 4): [(ops["create"], 1.0)],
            (4, 4): [(ops["ident"], 1.0)]}
    if V != 0.0:
        bulk[(0, 3)] = [(ops["count"], V)]
        bulk[(3, 4)] = [(ops["count"], 1.0)]
    herm = {0: 0, 1: 2, 2: 1, 3: 3, 4: 4}
    mpo = _fsm_mpo(L, 5, bulk, 0, 4, herm, {})
    N = L // 2 if N is None else N
    dense = [(U / 2, [(p, "interaction")]) for p in range(L)]
    for p in range(L - 1):
        dense += [(-t, [(p, "create"), (p + 1, "destroy")]), (-t, [(p, "destroy"), (p + 1, "create")])]
        if V != 0.0:
            dense.append((V, [(p, "count"), (p + 1, "count")]))
    return Model("bose_hubbard", capi.U1, phys, local, mpo, (N, 0), dense)


# ---- two-site MPO ---------------------------------------------------------------

def fuse_phys(p1, p2):
    """Two-site physical index and the offset of each (s1, s2) pair inside its
    fused sector (ProductBasis, indexing_stable.hpp:310-345: s1-major)."""
    sizes, order, offs = {}, [], {}
    for c1, d1 in p1:
        for c2, d2 in p2:
            f = (c1[0] + c2[0], c1[1] + c2[1])
            if f not in sizes:
                sizes[f] = 0
                order.append(f)
            offs[(c1, c2)] = sizes[f]
            sizes[f] += d1 * d2
    return [(f, sizes[f]) for f in order], offs


def kron_op(A: SiteOp, B: SiteOp, p1, p2) -> SiteOp:
    """Operator on the fused two-site basis, entry (i1*d2_in + i2, j1*d2_out + j2)."""
    phys12, offs = fuse_phys(p1, p2)
    d1, d2 = dict(p1), dict(p2)
    dims = dict(phys12)
    blocks = {}
    for (a_in, a_out), Ab in A.blocks.items():
        for (b_in, b_out), Bb in B.blocks.items():
            cin = (a_in[0] + b_in[0], a_in[1] + b_in[1])
            cout = (a_out[0] + b_out[0], a_out[1] + b_out[1])
            blk = blocks.setdefault((cin, cout), np.zeros((dims[cin], dims[cout])))
            ri, ro = offs[(a_in, b_in)], offs[(a_out, b_out)]
            for i1 in range(d1[a_in]):
                for i2 in range(d2[b_in]):
                    for j1 in range(d1[a_out]):
                        for j2 in range(d2[b_out]):
                            blk[ri + i1 * d2[b_in] + i2, ro + j1 * d2[b_out] + j2] += Ab[i1, j1] * Bb[i2, j2]
    blocks = {k: v for k, v in blocks.items() if np.any(v != 0)}
    return SiteOp(blocks=blocks, name=f"({A.name}x{B.name})")


def twosite_mpo(W1: MPOTensor, W2: MPOTensor, p1, p2, merge: bool = True) -> MPOTensor:
    """W12(b1, b3) = sum_b2 W1(b1, b2) x W2(b2, b3) (make_twosite_mpo, ts_ops.hpp:96-158):
    a single summand keeps its kron'd operator with the product of scales, several
    summands are added into one operator with scale 1.

    merge=False keeps every summand as its own (operator, s1 * s2) term -- the same
    operator sum -- and records in `sources[(b1, b3)]` the pair of site terms
    ((b1, b2, j1), (b2, b3, j2)) of each, so that derivatives with respect to the
    two-site term scales map back to the site MPO coefficients."""
    assert W1.col_dim == W2.row_dim
    terms = {}
    sources = {}
    # summands of every (b1, b3) in increasing b2, from the sparse entry lists
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
    for (b1, b3) in sorted(paths):
        summands = sorted(paths[(b1, b3)])
        if not merge:
            lst, src = [], []
            for b2 in summands:
                for j1, (o1, s1) in enumerate(W1.terms[(b1, b2)]):
                    for j2, (o2, s2) in enumerate(W2.terms[(b2, b3)]):
                        lst.append((kron_op(o1, o2, p1, p2), s1 * s2))
                        src.append(((b1, b2, j1), (b2, b3, j2)))
            terms[(b1, b3)] = lst
            sources[(b1, b3)] = src
            continue
        if len(summands) == 1 and len(W1.terms[(b1, summands[0])]) == 1 and len(W2.terms[(summands[0], b3)]) == 1:
            (o1, s1), = W1.terms[(b1, summands[0])]
            (o2, s2), = W2.terms[(summands[0], b3)]
            terms[(b1, b3)] = [(kron_op(o1, o2, p1, p2), s1 * s2)]
        else:
            acc = None
            for b2 in summands:
                for o1, s1 in W1.terms[(b1, b2)]:
                    for o2, s2 in W2.terms[(b2, b3)]:
                        k = kron_op(o1, o2, p1, p2)
                        k = SiteOp({kk: vv * (s1 * s2) for kk, vv in k.blocks.items()}, name=k.name)
                        if acc is None:
                            acc = k
                        else:
                            for kk, vv in k.blocks.items():
                                acc.blocks[kk] = acc.blocks.get(kk, 0) + vv
            acc.blocks = {k: v for k, v in acc.blocks.items() if np.any(v != 0)}
            if acc.blocks:
                terms[(b1, b3)] = [(acc, 1.0)]
    W = MPOTensor(W1.row_dim, W2.col_dim, terms, W1.left_herm, W1.left_phase, W2.right_herm, W2.right_phase,
                  W1.left_spin, W2.right_spin)
    if not merge:
        W.sources = sources
    return W


def twosite_for(model: Model, i: int, merge: bool = True) -> MPOTensor:
    """The two-site MPO of sites (i, i+1) of a model: the spin-coupled product for SU2U1
    (su2u1.twosite_mpo), the Kronecker product otherwise."""
    if model.symm == capi.SU2U1:
        from . import su2u1
        return su2u1.twosite_mpo(model.mpo[i], model.mpo[i + 1], model.phys, model.phys)
    return twosite_mpo(model.mpo[i], model.mpo[i + 1], model.phys, model.phys, merge=merge)


# ---- C description ------------------------------------------------------------------

class MPOHandle:
    """An MPO tensor registered with libdmrgb200 (dmrgb200_mpo_create)."""

    def __init__(self, W: MPOTensor, symm: int):
        ops, op_ids = [], {}
        tb1, tb2, top, tsc = [], [], [], []
        self.term_keys = []   # (b1, b2, j) of each described term, in description order
        for (b1, b2) in sorted(W.terms):
            for j, (op, sc) in enumerate(W.terms[(b1, b2)]):
                self.term_keys.append((b1, b2, j))
                if id(op) not in op_ids:
                    op_ids[id(op)] = len(ops)
                    ops.append(op)
                tb1.append(b1)
                tb2.append(b2)
                top.append(op_ids[id(op)])
                tsc.append(sc)
        op_block, blk_in, blk_out, blk_entry = [0], [], [], [0]
        e_row, e_col, e_rs, e_cs, e_coeff = [], [], [], [], []
        su2 = symm == capi.SU2U1
        for op in ops:
            for (cin, cout), B in op.blocks.items():
                blk_in += list(cin)
                blk_out += list(cout)
                if su2 and op.spins is not None:
                    rsp, csp = op.spins[(cin, cout)]
                elif su2:  # site operator: the entries' spins are those of the block's charges
                    rsp, csp = [abs(cin[1])] * B.shape[0], [abs(cout[1])] * B.shape[1]
                else:
                    rsp, csp = [0] * B.shape[0], [0] * B.shape[1]
                for i in range(B.shape[0]):
                    for j in range(B.shape[1]):
                        if B[i, j] != 0:
                            e_row.append(i)
                            e_col.append(j)
                            e_rs.append(rsp[i])
                            e_cs.append(csp[j])
                            e_coeff.append(B[i, j])
                blk_entry.append(len(e_row))
            op_block.append(len(blk_entry) - 1)
        none = 0xFFFFFFFF
        A = lambda v, dt: np.ascontiguousarray(np.array(v, dtype=dt))
        self._keep = dict(
            term_b1=A(tb1, np.uint32), term_b2=A(tb2, np.uint32), term_op=A(top, np.uint32),
            term_scale=A(tsc, np.float64), op_spin=A([o.spin for o in ops], np.int32),
            op_block=A(op_block, np.uint32), blk_in=A(blk_in, np.int32), blk_out=A(blk_out, np.int32),
            blk_entry=A(blk_entry, np.uint32), e_row=A(e_row, np.uint32), e_col=A(e_col, np.uint32),
            e_row_spin=A(e_rs, np.int32), e_col_spin=A(e_cs, np.int32), e_coeff=A(e_coeff, np.float64),
            left_herm=A([none if h is None else h for h in W.left_herm] if W.left_herm else [], np.uint32),
            left_phase=A(W.left_phase or [], np.int32),
            right_herm=A([none if h is None else h for h in W.right_herm] if W.right_herm else [], np.uint32),
            right_phase=A(W.right_phase or [], np.int32),
            left_spin=A(W.left_spin or [], np.int32), right_spin=A(W.right_spin or [], np.int32))
        k = self._keep
        d = capi.MpoDesc()
        d.symm = symm
        d.row_dim, d.col_dim = W.row_dim, W.col_dim
        d.left_spin = capi.ptr(k["left_spin"], capi.C.c_int32) if W.left_spin else None
        d.right_spin = capi.ptr(k["right_spin"], capi.C.c_int32) if W.right_spin else None
        d.left_herm = capi.ptr(k["left_herm"], capi.C.c_uint32) if W.left_herm else None
        d.left_phase = capi.ptr(k["left_phase"], capi.C.c_int32) if W.left_herm else None
        d.right_herm = capi.ptr(k["right_herm"], capi.C.c_uint32) if W.right_herm else None
        d.right_phase = capi.ptr(k["right_phase"], capi.C.c_int32) if W.right_herm else None
        d.n_terms = len(tb1)
        d.term_b1 = capi.ptr(k["term_b1"], capi.C.c_uint32)
        d.term_b2 = capi.ptr(k["term_b2"], capi.C.c_uint32)
        d.term_op = capi.ptr(k["term_op"], capi.C.c_uint32)
        d.term_scale = capi.ptr(k["term_scale"], capi.C.c_double)
        d.n_ops = len(ops)
        d.op_spin = capi.ptr(k["op_spin"], capi.C.c_int32)
        d.op_block = capi.ptr(k["op_block"], capi.C.c_uint32)
        d.blk_in = capi.ptr(k["blk_in"], capi.C.c_int32)
        d.blk_out = capi.ptr(k["blk_out"], capi.C.c_int32)
        d.blk_entry = capi.ptr(k["blk_entry"], capi.C.c_uint32)
        d.e_row = capi.ptr(k["e_row"], capi.C.c_uint32)
        d.e_col = capi.ptr(k["e_col"], capi.C.c_uint32)
        d.e_row_spin = capi.ptr(k["e_row_spin"], capi.C.c_int32)
        d.e_col_spin = capi.ptr(k["e_col_spin"], capi.C.c_int32)
        d.e_coeff = capi.ptr(k["e_coeff"], capi.C.c_double)
        h = capi.C.c_void_p()
        capi.check(capi.lib.dmrgb200_mpo_create(capi.C.byref(d), capi.C.byref(h)), "dmrgb200_mpo_create")
        self.handle = h
        self.row_dim, self.col_dim = W.row_dim, W.col_dim
        self.term_scale = np.array(tsc, dtype=np.float64)
        self.n_terms = len(tsc)

    def __del__(self):
        if getattr(self, "handle", None):
            capi.lib.dmrgb200_mpo_destroy(self.handle)
            self.handle = None
