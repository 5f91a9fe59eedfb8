"""Derivatives of E = <psi|H|psi> with respect to the one- and two-electron integrals
of a quantum-chemistry MPO for a whole MPS -- 1-/2-RDM elements -- by moving the
two-site centre over every site pair.

An integral's coefficient sits in the MPO tensors of one or more sites.  With the
state in mixed-canonical form at sites (i, i+1), E = <Theta|H_eff|Theta>, and the
part of dE/dc that comes from the coefficients in W_i (and, at the last pair, in
W_{i+1}) is exact there: H_eff is linear in the terms of the two-site MPO, whose
scales are linear in each site's coefficients, so it is galpha . d alpha / dc with
galpha = d<Theta|H_eff Theta>/d alpha from the adjoint (dmrgb200_hpsi_adjoint) and
d alpha / dc read off the plan of the MPO with the integral raised by one in that
site tensor only.  Summing the parts over the sites gives the full derivative for
the normalised state, including integrals whose coefficients live in the boundaries
of any one centre.  The centre moves by exact (untruncated) SVD splits and left
boundary steps, so the state is the same at every pair.

The reference measures RDM elements by contracting operator MPOs over the chain
(models/measurements/tagged_nrankrdm.h:91-411); here they are derivatives of the
energy, the reference's H being the product of the same site tensors.
"""
from __future__ import annotations

import numpy as np

from . import _capi as capi
from . import dmrg as G
from . import engine as E
from . import models as M
from . import qc


def _twosite(W1, W2, model):
    """Two-site MPO whose term scales are linear in each site's scales: the spin-coupled
    product for SU2U1, the unmerged Kronecker product otherwise."""
    if model.symm == capi.SU2U1:
        from . import su2u1
        return su2u1.twosite_mpo(W1, W2, model.phys, model.phys)
    return M.twosite_mpo(W1, W2, model.phys, model.phys, merge=False)


def _alpha(p12, left, right, W1, W2, model, Lidx, Ridx):
    W12 = M.MPOHandle(_twosite(W1, W2, model), model.symm)
    return E.schedule_hpsi(p12, left, right, W12, Lidx, Ridx).plan


def with_integrals(model, h, eri):
    """The quantum-chemistry model of `model`'s kind (TwoU1 or SU2U1), sites and electrons
    with other integrals."""
    L = len(model.mpo)
    if model.symm == capi.SU2U1:
        from . import su2u1
        return su2u1.quantum_chemistry(L, model.total_charge[0], model.total_charge[1], h=h, eri=eri)
    return qc.quantum_chemistry(L, model.total_charge[0], model.total_charge[1], h=h, eri=eri)


def integral_derivatives(backend, model, tensors, integrals) -> dict:
    """dE/dc for every c in `integrals` (("h", (a, b)) or ("eri", (a, b, c, d)); the
    orbit of the index as qc.raise_integral raises it) of the quantum-chemistry model
    (TwoU1, or SU2U1 where H_eff acts on the spin-reduced two-site tensor) for the
    normalised state of `tensors`.  backend: an object with edge, left_step, right_step
    (as dmrg.DeviceBackend / the oracle backend) and galpha(plan, Lidx, Lbuf, Ridx, Rbuf,
    x) returning d<x|H x>/d alpha per plan term."""
    L = len(tensors)
    su2 = model.symm == capi.SU2U1
    raised = {key: with_integrals(model, *qc.raise_integral(model.h, model.eri, key[0], key[1], 1.0))
              for key in integrals}
    A = G.right_canonicalize(list(tensors), 0.0)
    p12, offs = M.fuse_phys(model.phys, model.phys)
    W = [M.MPOHandle(w, model.symm) for w in model.mpo]
    Lidx, Lbuf = backend.edge(model.symm, A[0].left)
    R = [None] * (L + 1)
    R[L] = backend.edge(model.symm, A[-1].right)
    for j in range(L - 1, 1, -1):
        R[j] = backend.right_step(model, W[j], R[j + 1][0], R[j + 1][1], A[j])
    out = {key: 0.0 for key in integrals}
    norm = None
    for i in range(L - 1):
        psi = G.twosite(A[i], A[i + 1], p12, offs)
        if norm is None:
            norm = float(np.linalg.norm(psi.data))
        psi.data = psi.data / norm
        Ridx, Rbuf = R[i + 2]
        base = _alpha(p12, psi.left, psi.right, model.mpo[i], model.mpo[i + 1], model, Lidx, Ridx)
        if su2:
            # H_eff acts on the spin-reduced two-site tensor (the 6j recoupling is orthogonal)
            from . import su2u1
            x = su2u1.reduce_twosite(psi, model.phys, model.phys, offs).data
        else:
            x = psi.data
        ga = backend.galpha(base, Lidx, Lbuf, Ridx, Rbuf, x)
        sites = (i, i + 1) if i == L - 2 else (i,)
        for key, m2 in raised.items():
            for j in sites:
                W1 = m2.mpo[i] if j == i else model.mpo[i]
                W2 = m2.mpo[i + 1] if j == i + 1 else model.mpo[i + 1]
                plan = _alpha(p12, psi.left, psi.right, W1, W2, model, Lidx, Ridx)
                for k in ("term_t", "term_col", "l_term", "l_b1"):
                    if not np.array_equal(base[k], plan[k]):
                        raise ValueError("the MPO structure changes with the integral value")
                out[key] += float(np.asarray(ga) @ (plan["term_alpha"] - base["term_alpha"]))
        if i < L - 2:
            res = G.split(psi, model.phys, model.phys, offs, 10 ** 9, 0.0, True)
            A[i], A[i + 1] = res.A, res.B
            A[i + 1].data = A[i + 1].data * norm
            Lidx, Lbuf = backend.left_step(model, W[i], Lidx, Lbuf, A[i])
    return out
