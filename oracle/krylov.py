"""Oracle: Krylov solvers of the SolverV4 path (TEST INFRASTRUCTURE)."""

from __future__ import annotations

import numpy as np


def pcg(A, b, M, x0=None, tol=1e-5, maxiter=1000, history=None):
    """Preconditioned CG with the reference's up-front convergence check
    (solver_v2.py:552-624). ``iters`` counts preconditioner applications.
    Returns (x, iters, converged)."""
    x = np.zeros_like(b) if x0 is None else x0.copy()
    r = b - A(x)
    bb = float(np.dot(b, b))
    tol_sq = tol**2 * bb
    rr0 = float(np.dot(r, r))
    if history is not None:
        history.append((rr0 / bb) ** 0.5 if bb > 0 else 0.0)
    if rr0 <= tol_sq:
        return x, 0, True
    z = M(r)
    p = z.copy()
    rz = float(np.dot(r, z))
    iters = 1
    for _ in range(maxiter - 1):
        Ap = A(p)
        alpha = rz / float(np.dot(p, Ap))
        x = x + alpha * p
        r = r - alpha * Ap
        rr = float(np.dot(r, r))
        if history is not None:
            history.append((rr / bb) ** 0.5 if bb > 0 else 0.0)
        if rr <= tol_sq:
            return x, iters, True
        z = M(r)
        iters += 1
        rz_new = float(np.dot(r, z))
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x, iters, False


def fgmres(A, b, M, x0=None, tol=1e-6, maxiter=200, restart=32, history=None):
    """Right-preconditioned restarted flexible GMRES with modified Gram-Schmidt
    and Givens rotations (multigrid_v4.py:325-443). Returns (x, iters, converged)."""
    x = np.zeros_like(b) if x0 is None else x0.copy()
    bn = float(np.linalg.norm(b))
    if bn <= 1e-30:
        return x, 0, True
    total = 0
    converged = False
    while total < maxiter:
        r = b - A(x)
        beta = float(np.linalg.norm(r))
        if history is not None:
            history.append(beta / bn)
        if beta / bn <= tol:
            converged = True
            break
        V = [r / beta]
        Z = []
        H = np.zeros((restart + 1, restart))
        cs = np.zeros(restart)
        sn = np.zeros(restart)
        g = np.zeros(restart + 1)
        g[0] = beta
        jf = 0
        for j in range(min(restart, maxiter - total)):
            z = M(V[j])
            Z.append(z)
            w = A(z)
            for i in range(j + 1):
                H[i, j] = float(np.dot(V[i], w))
                w = w - H[i, j] * V[i]
            H[j + 1, j] = float(np.linalg.norm(w))
            hn = H[j + 1, j]
            if hn > 1e-14:
                V.append(w / hn)
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            den = np.sqrt(H[j, j] ** 2 + H[j + 1, j] ** 2)
            cs[j], sn[j] = (1.0, 0.0) if den < 1e-300 else (H[j, j] / den, H[j + 1, j] / den)
            H[j, j] = cs[j] * H[j, j] + sn[j] * H[j + 1, j]
            H[j + 1, j] = 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            total += 1
            jf = j + 1
            if history is not None:
                history.append(abs(g[j + 1]) / bn)
            if abs(g[j + 1]) / bn <= tol or hn <= 1e-14:
                converged = True
                break
        if jf > 0:
            R = np.triu(H[:jf, :jf])
            try:
                y = np.linalg.solve(R, g[:jf].copy())
            except np.linalg.LinAlgError:
                y = np.linalg.lstsq(R, g[:jf].copy(), rcond=None)[0]
            for c, z in zip(y, Z[:jf]):
                x = x + float(c) * z
        if converged:
            break
    return x, total, converged
