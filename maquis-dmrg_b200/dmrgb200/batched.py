"""Jacobi-Davidson on many independent site problems at once.

The instances share one batched plan (dmrgb200_plan_create_batched: every H·psi
stage is one launch over the tiles of all instances) and one batched vector in
which instance i occupies [in_base[i], in_base[i] + size_i).  Each iteration
runs the steps of the reference's solver (ietl/jacobi.h:386-474 with
ietl_jcd_gmres = 0; the same steps as dmrgb200_solve and oracle/jd.py) for every
instance independently: the vector operations are segment reductions over the
batched vector (one kernel for all instances), the Rayleigh-Ritz problems a
batch of small symmetric eigenproblems, and the H·psi one batched product in
FP64 or emulated FP64.  No counterpart in the reference, which solves one site
problem at a time."""
from __future__ import annotations

import numpy as np

from . import _capi as capi


class BatchedJD:
    def __init__(self, plan, device="cuda"):
        """plan: engine.BatchedPlan."""
        import torch
        self.torch, self.plan = torch, plan
        self.n = len(plan.in_base)
        self.total = int(plan.total_size)
        seg = np.zeros(self.total, dtype=np.int64)
        for i, b in enumerate(plan.in_base):
            seg[b:] = i  # padding after an instance belongs to it (it stays zero)
        self.seg = torch.from_numpy(seg).to(device)
        self.device = device

    def _dot(self, a, b):
        out = self.torch.zeros(self.n, dtype=a.dtype, device=a.device)
        return out.index_add_(0, self.seg, a * b)

    def _scale(self, coef):  # per-instance coefficient -> per element
        return coef[self.seg]

    def solve(self, x0, max_iter: int = 20, tol: float = 0.0, prec: int = capi.PREC_FP64, stream: int = 0):
        """Lowest eigenpair of every instance from the start vectors x0 (batched layout,
        zero padding).  Returns (theta[n], u batched vector, iterations[n], residual norms[n]);
        an instance stops when |r| <= tol |theta| or |r| < tol (iteration.h:56-58), the
        others continue (tol 0: every instance runs max_iter iterations)."""
        torch = self.torch
        kappa = 0.25
        V, VA = [], []
        M = torch.zeros((self.n, max_iter, max_iter), dtype=torch.float64, device=x0.device)
        active = torch.ones(self.n, dtype=torch.bool, device=x0.device)
        iters = torch.zeros(self.n, dtype=torch.int64, device=x0.device)
        theta = torch.zeros(self.n, dtype=torch.float64, device=x0.device)
        rn = torch.zeros_like(theta)
        u = x0.clone()
        t = x0.clone()
        for it in range(max_iter):
            tau = torch.sqrt(self._dot(t, t))
            for v in V:
                t = t - self._scale(self._dot(v, t)) * v
            again = torch.sqrt(self._dot(t, t)) < kappa * tau
            if bool(again.any()):
                t2 = t
                for v in V:
                    t2 = t2 - self._scale(self._dot(v, t2)) * v
                t = torch.where(self._scale(again), t2, t)
            t = t / self._scale(torch.sqrt(self._dot(t, t)))
            y = torch.zeros_like(t)
            self.plan.hpsi(t.data_ptr(), y.data_ptr(), prec, stream)
            V.append(t)
            VA.append(y)
            for i in range(it + 1):
                M[:, i, it] = self._dot(V[i], y)
            k = it + 1
            Mk = torch.triu(M[:, :k, :k]) + torch.triu(M[:, :k, :k], 1).transpose(1, 2)
            w, z = torch.linalg.eigh(Mk)
            th, s = w[:, 0], z[:, :, 0]
            un = torch.zeros_like(t)
            uA = torch.zeros_like(t)
            for j in range(k):
                cj = self._scale(s[:, j])
                un = un + cj * V[j]
                uA = uA + cj * VA[j]
            r = uA - self._scale(th) * un
            rr = torch.sqrt(self._dot(r, r))
            # instances still iterating take this iteration's results
            theta = torch.where(active, th, theta)
            rn = torch.where(active, rr, rn)
            u = torch.where(self._scale(active), un, u)
            iters = iters + active.to(torch.int64)
            done = (rr <= tol * th.abs()) | (rr < tol)
            active = active & ~done
            if not bool(active.any()) or it + 1 >= max_iter:
                break
            t = -r + self._scale(self._dot(r, un) / self._dot(un, un)) * un
        return theta, u, iters, rn
