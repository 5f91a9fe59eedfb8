"""ORACLE — test infrastructure only.  CPU backend of the two-site sweep driver
(dmrgb200.dmrg.TwoSiteDMRG): boundary steps and H·psi by the oracle's
restatement of the reference's schedule execution, eigenpairs by the numpy
restatement of the reference's Jacobi-Davidson (jd.py), so that a whole sweep
can be replayed on the CPU and compared with the device sweep."""
from __future__ import annotations

import jd as JD
import oracle as O
from dmrgb200 import engine as E


class OracleBackend:
    def edge(self, symm, index):
        idx = E.edge_bindex(symm, index)
        return idx, idx.edge_values()

    def left_step(self, model, W, Lidx, Lval, t):
        sch, nidx = E.schedule_left_step(model.phys, t.left, t.right, W, Lidx, True)
        return nidx, O.left_step(sch.plan, Lval, Lidx, t.data, t.left_paired(), nidx)

    def right_step(self, model, W, Ridx, Rval, t):
        sch, nidx = E.schedule_right_step(model.phys, t.left, t.right, W, Ridx, True)
        return nidx, O.right_step(sch.plan, Rval, Ridx, t.data, t.data, nidx)

    def alpha_dm(self, phys, W, idx, val, t, alpha, left):
        if left:
            sch, _ = E.schedule_left_step(phys, t.left, t.right, W, idx, False)
            return O.alpha_dm(sch.plan, val, idx, t.data, t.left_paired(), alpha)
        sch, _ = E.schedule_right_step(phys, t.left, t.right, W, idx, False)
        return O.alpha_dm(sch.plan, val, idx, t.data, t.data, alpha)

    def galpha(self, plan, Lidx, Lval, Ridx, Rval, x):
        return O.hpsi_adjoint(plan, Lval, Lidx, Rval, Ridx, x, x)[1]

    def solve(self, p12, psi, W12, Lidx, Lval, Ridx, Rval, tol, max_iter):
        sch = E.schedule_hpsi(p12, psi.left, psi.right, W12, Lidx, Ridx)
        theta, u, it, conv, rn = JD.jcd(lambda v: O.hpsi(sch.plan, Lval, Lidx, Rval, Ridx, v), psi.data, tol=tol,
                                        max_iter=max_iter)
        return theta, u, it, 0.0

    def sync(self):
        pass
