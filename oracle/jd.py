"""ORACLE — test infrastructure only.  numpy restatement of the reference's
Jacobi-Davidson solver with ietl_jcd_gmres = 0:
  solve_ietl_jcd          dmrg/framework/dmrg/solver/ietl_jacobi_davidson.h:35-76
  calculate_eigenvalue    dmrg/framework/ietl/jacobi.h:386-474 (MGS + refinement,
                          Rayleigh-Ritz smallest pair, residual, correction :141-157)
  basic_iteration         dmrg/framework/ietl/iteration.h:41-78
"""
from __future__ import annotations

import numpy as np


def jcd(matvec, x0: np.ndarray, ortho=(), tol: float = 1e-8, max_iter: int = 8):
    ortho = [np.array(o, dtype=np.float64) for o in ortho]
    for n in range(1, len(ortho)):
        for n0 in range(n):
            ortho[n] = ortho[n] - ortho[n0].dot(ortho[n]) / ortho[n0].dot(ortho[n0]) * ortho[n0]

    def project(t):
        for o in ortho:
            t = t - o.dot(t) / o.dot(o) * o
        return t

    V = [None] * max_iter
    VA = [None] * max_iter
    M = np.zeros((max_iter, max_iter))
    kappa = 0.25
    V[0] = project(np.array(x0, dtype=np.float64))
    it = 0
    while True:
        t = V[it]
        tau = np.linalg.norm(t)
        for i in range(1, it + 1):
            t = t - V[i - 1].dot(t) * V[i - 1]
        if np.linalg.norm(t) < kappa * tau:
            for i in range(1, it + 1):
                t = t - V[i - 1].dot(t) * V[i - 1]
        t = project(t)
        t = t / np.linalg.norm(t)
        V[it] = t
        VA[it] = matvec(t)
        for i in range(it + 1):
            M[i, it] = V[i].dot(VA[it])
        k = it + 1
        Mk = np.triu(M[:k, :k]) + np.triu(M[:k, :k], 1).T
        w, z = np.linalg.eigh(Mk)
        theta, s = w[0], z[:, 0]
        u = V[0] * s[0]
        for j in range(1, k):
            u = u + V[j] * s[j]
        uA = VA[0] * s[0]
        for j in range(1, k):
            uA = uA + VA[j] * s[j]
        uA = project(uA)
        r = uA - theta * u
        it += 1
        rn = np.linalg.norm(r)
        if rn <= tol * abs(theta) or rn < tol:
            return theta, u, it, True, rn
        if it >= max_iter:
            return theta, u, it, False, rn
        V[it] = -r + r.dot(u) / u.dot(u) * u
