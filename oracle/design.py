"""Oracle: design update (OC) and density filter (TEST INFRASTRUCTURE)."""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp


def oc_update(rho, dc, volfrac, move=0.10, rho_min=1e-3):
    """Bisection OC of the public GPU path (topogpu/solver.py:94-117).

    lambda_hi doubles from 1 while the candidate's mean exceeds volfrac (and
    lambda_hi < 1e40); then up to 80 bisections, stopping early once
    |mean - volfrac| < 1e-8. Returns the LAST candidate evaluated, plus the
    number of candidate evaluations (doubling + bisection).
    """
    rho = np.asarray(rho, dtype=np.float64)
    dcs = np.minimum(np.asarray(dc, dtype=np.float64), -1.0e-12)
    lo_b = np.maximum(rho - move, rho_min)
    hi_b = np.minimum(rho + move, 1.0)

    def cand(lam):
        return np.clip(rho * np.sqrt(np.maximum(-dcs / max(lam, 1.0e-40), 0.0)), lo_b, hi_b)

    lam_lo, lam_hi = 0.0, 1.0
    n_eval = 0
    while True:
        n_eval += 1
        if not (cand(lam_hi).mean() > volfrac and lam_hi < 1.0e40):
            break
        lam_lo = lam_hi
        lam_hi *= 2.0
    new = None
    for _ in range(80):
        mid = 0.5 * (lam_lo + lam_hi)
        new = cand(mid)
        n_eval += 1
        m = new.mean()
        if m > volfrac:
            lam_lo = mid
        else:
            lam_hi = mid
        if abs(float(m) - volfrac) < 1.0e-8:
            break
    return new, n_eval


def filter_offsets(rmin: float):
    """Integer offsets (dx,dy,dz) and weights of the linear-hat filter.

    The reference pairs elements whose centre distance is at most rmin-1e-10
    (kd-tree ``query_pairs``, pub_simp_solver.py:225-236), weight rmin - d,
    and adds each element to itself with weight rmin. On a unit grid that is
    the fixed stencil returned here (order: dx, dy, dz ascending).
    """
    R = int(math.floor(rmin))
    out = []
    for dx in range(-R, R + 1):
        for dy in range(-R, R + 1):
            for dz in range(-R, R + 1):
                d = math.sqrt(float(dx * dx + dy * dy + dz * dz))
                if dx == dy == dz == 0:
                    out.append((0, 0, 0, rmin))
                elif d <= rmin - 1e-10:
                    out.append((dx, dy, dz, rmin - d))
    return out


def filter_matrix(nel, rmin: float) -> sp.csr_matrix:
    """Row-normalised H (pub_simp_solver.py:215-243), as CSR."""
    nx, ny, nz = nel
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ix, iy, iz = ix.ravel(), iy.ravel(), iz.ravel()
    n = nx * ny * nz
    rows, cols, w = [], [], []
    for dx, dy, dz, wt in filter_offsets(rmin):
        jx, jy, jz = ix + dx, iy + dy, iz + dz
        ok = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny) & (jz >= 0) & (jz < nz)
        rows.append(np.nonzero(ok)[0])
        cols.append(((jx * ny + jy) * nz + jz)[ok])
        w.append(np.full(int(ok.sum()), wt))
    rows, cols, w = np.concatenate(rows), np.concatenate(cols), np.concatenate(w)
    Hs = np.zeros(n)
    np.add.at(Hs, rows, w)
    return sp.csr_matrix((w / Hs[rows], (rows, cols)), shape=(n, n))


def dense_filter_matrix(nel, radius: float) -> np.ndarray:
    """DensityFilter.matrix (topogpu/filter.py:14-29): dense max(0, r - d), row-normalised."""
    nx, ny, nz = nel
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    c = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1).astype(float)
    d = np.linalg.norm(c[:, None, :] - c[None, :, :], axis=2)
    w = np.maximum(0.0, radius - d)
    s = w.sum(axis=1)
    s[s == 0.0] = 1.0
    return w / s[:, None]


def oc_update_filtered(rho, dc, dv, volfrac, move, H, rho_min=1e-3):
    """Filtered-volume OC of ``run_simp`` (pub_simp_solver.py:319-340), no
    Heaviside: l1=0, l2=1e9, <=100 bisections, stop when l2-l1 < 1e-9; the
    volume is measured on H*candidate. Returns (candidate, n_eval)."""
    rho = np.asarray(rho, dtype=np.float64)
    dcs = np.minimum(dc, -1e-12)
    dvs = np.maximum(dv, 1e-12)
    n = len(rho)
    l1, l2 = 0.0, 1e9
    rn = None
    k = 0
    for k in range(100):
        lm = 0.5 * (l1 + l2)
        rn = rho * np.sqrt(-dcs / (lm * dvs))
        rn = np.clip(rn, rho - move, rho + move)
        rn = np.clip(rn, rho_min, 1.0)
        if (H @ rn).sum() / n > volfrac:
            l1 = lm
        else:
            l2 = lm
        if l2 - l1 < 1e-9:
            break
    return rn, k + 1


def heaviside(rho_f, beta, eta):
    """Smoothed Heaviside projection of run_simp (pub_simp_solver.py:245-248):
    (tanh(b e) + tanh(b (x - e))) / (tanh(b e) + tanh(b (1 - e))); identity
    for beta < 1e-6."""
    rho_f = np.asarray(rho_f, dtype=np.float64)
    if beta < 1e-6:
        return rho_f.copy()
    return (np.tanh(beta * eta) + np.tanh(beta * (rho_f - eta))) / (np.tanh(beta * eta) + np.tanh(beta * (1.0 - eta)))


def heaviside_deriv(rho_f, beta, eta):
    """d heaviside / d rho_f (pub_simp_solver.py:250-253)."""
    rho_f = np.asarray(rho_f, dtype=np.float64)
    if beta < 1e-6:
        return np.ones_like(rho_f)
    denom = np.tanh(beta * eta) + np.tanh(beta * (1.0 - eta))
    return beta * (1.0 - np.tanh(beta * (rho_f - eta)) ** 2) / denom


def oc_update_projected(rho, dc, dv, volfrac, move, H, beta, eta, rho_min=1e-3):
    """run_simp's OC with the volume measured after filter AND Heaviside
    projection (pub_simp_solver.py:319-340 with use_heaviside and beta >
    1e-6): l1=0, l2=1e9, <=100 bisections, stop when l2-l1 < 1e-9. Returns
    (candidate, n_eval)."""
    rho = np.asarray(rho, dtype=np.float64)
    dcs = np.minimum(dc, -1e-12)
    dvs = np.maximum(dv, 1e-12)
    n = len(rho)
    l1, l2 = 0.0, 1e9
    rn = None
    k = 0
    for k in range(100):
        lm = 0.5 * (l1 + l2)
        rn = rho * np.sqrt(-dcs / (lm * dvs))
        rn = np.clip(rn, rho - move, rho + move)
        rn = np.clip(rn, rho_min, 1.0)
        if heaviside(H @ rn, beta, eta).sum() / n > volfrac:
            l1 = lm
        else:
            l2 = lm
        if l2 - l1 < 1e-9:
            break
    return rn, k + 1


def grayness(rho) -> float:
    """4 mean(rho(1-rho)) (topogpu/solver.py:120-121)."""
    rho = np.asarray(rho)
    return float(4.0 * np.mean(rho * (1.0 - rho)))
