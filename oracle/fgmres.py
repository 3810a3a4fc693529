"""CPU oracle of flexible GMRES (test infrastructure only).

The reference has no flexible GMRES: this restates the published algorithm
(Y. Saad, "A flexible inner-outer preconditioned GMRES algorithm", SIAM J.
Sci. Comput. 14 (1993) 461-469; Saad, Iterative Methods for Sparse Linear
Systems, 2nd ed., Algorithm 9.6) with the restart and termination rules of
the reference's GMRES (linalg/GMRES.java:40-251):

* absolute tolerance on |gamma_{j+1}| (the Givens residual estimate), a cycle
  ends when it drops below ``tol`` or when ``j > restart``
  (GMRES.java:170, the inner loop keeps going one column past IBR);
* after each cycle x += Z y (y from the triangular solve of calculateAlpha,
  GMRES.java:239-251); the method restarts when the cycle ran past
  ``restart`` columns or the true residual ||b - A x|| is above ``tol``
  (GMRES.java:92), at most ``max_restarts`` times;
* the iteration counter advances only when the cycle continues, so the last
  estimate of a cycle is overwritten by the first of the next one.

Orthogonalisation is classical Gram-Schmidt applied twice (CGS2), as in the
CUDA path.  Pure numpy, for systems of a few thousand unknowns.
"""
from __future__ import annotations

import numpy as np

OK, MAXITER, NONFINITE = 0, 1, 3


def solve_fgmres(matvec, precond, b, tol, x0=None, restart=30, max_restarts=200):
    """Returns (x, iterations, restarts, status, history)."""
    b = np.asarray(b, dtype=np.float64)
    n = b.size
    x = np.zeros(n) if x0 is None else np.asarray(x0, dtype=np.float64).copy()
    it = 0
    restarts = 0
    hist = {}
    ldh = restart + 10
    status = MAXITER
    while True:
        r = b - matvec(x)
        g0 = float(np.sqrt(r @ r))
        if not np.isfinite(g0):
            status = NONFINITE
            break
        if g0 <= tol:
            status = OK
            break
        H = np.zeros((ldh, ldh))
        gam = np.zeros(ldh)
        cs = np.zeros(ldh)
        sn = np.zeros(ldh)
        gam[0] = g0
        V = [r / g0]
        Z = []
        j = 0
        jfin = 0
        bad = False
        while True:
            z = precond(V[j])
            Z.append(z)
            t = matvec(z)
            Vm = np.array(V)
            f1 = Vm @ t
            w = t - Vm.T @ f1
            f2 = Vm @ w
            w = w - Vm.T @ f2
            H[:j + 1, j] += f1 + f2
            H[j + 1, j] += np.sqrt(w @ w)
            for i in range(j):
                hij, hipj = H[i, j], H[i + 1, j]
                H[i, j] = hij * cs[i] + hipj * sn[i]
                H[i + 1, j] = -hij * sn[i] + hipj * cs[i]
            hjj, hj1 = H[j, j], H[j + 1, j]
            beta = np.sqrt(hjj * hjj + hj1 * hj1)
            sn[j] = hj1 / beta
            cs[j] = hjj / beta
            H[j, j] = beta
            gam[j + 1] = -sn[j] * gam[j]
            gam[j] = cs[j] * gam[j]
            g = abs(gam[j + 1])
            hist[it] = g
            if g < tol or j > restart or not np.isfinite(g):
                jfin = j
                bad = not np.isfinite(g)
                break
            V.append(w / H[j + 1, j])
            it += 1
            j += 1
            if j == n:
                jfin = n - 1
                break
        if bad:
            status = NONFINITE
            break
        alpha = np.zeros(jfin + 1)
        for i in range(jfin, -1, -1):
            s = H[i, i + 1:jfin + 1] @ alpha[i + 1:jfin + 1]
            alpha[i] = 1.0 / H[i, i] * (gam[i] - s)
        x = x + np.array(Z[:jfin + 1]).T @ alpha
        rt = b - matvec(x)
        true_res = float(np.sqrt(rt @ rt))
        if not np.isfinite(true_res):
            status = NONFINITE
            break
        if (jfin > restart and restarts < max_restarts) or true_res > tol:
            if restarts < max_restarts:
                restarts += 1
                continue
            status = MAXITER
            break
        status = OK
        break
    h = np.array([hist[i] for i in range(it)]) if it > 0 else np.zeros(0)
    return x, it, restarts, status, h
