"""Oracle: Galerkin geometric multigrid of SolverV4 (TEST INFRASTRUCTURE).

Restates ``GalerkinMatFreeGMG`` (reference ``src/gpu_fem/multigrid_v4.py:446-1042``)
and its helpers from ``src/gpu_fem/solver_v2.py`` on compact free-DoF vectors
with SciPy CSR, exactly as the reference arranges them.
"""

from __future__ import annotations

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

from . import fem


def level_dims(nel, n_levels: int):
    """multigrid_v4.py:525-529: each level halves, floored, never below 1."""
    dims = [tuple(nel)]
    for _ in range(1, n_levels):
        dims.append(tuple(max(1, d // 2) for d in dims[-1]))
    return dims


def _weights_1d(nf: int, nc: int):
    """1-D trilinear parent weights, row-normalised (solver_v2.py:62-149).

    Fine node i (0..nf) takes parent i//2 (+1 when i is odd) with weight 1
    (even) or 1/2 (odd); parents beyond nc drop out and the row is scaled so
    it sums to one. Returns a list of [(parent, weight), ...] per fine node.
    """
    out = []
    for i in range(nf + 1):
        cand = [(i >> 1, 1.0)] if (i & 1) == 0 else [(i >> 1, 0.5), ((i >> 1) + 1, 0.5)]
        cand = [(c, w) for c, w in cand if 0 <= c <= nc]
        s = sum(w for _, w in cand)
        out.append([(c, w / s) for c, w in cand])
    return out


def scalar_prolongation(fine, coarse) -> sp.csr_matrix:
    """Node-to-node trilinear P (n_fine_nodes x n_coarse_nodes), rows sum to 1.

    The reference builds the raw tensor-product weights and then scales each
    row by 1/rowsum (solver_v2.py:135-148). Per-dimension validity makes the
    row sum a product of 1-D sums, so the normalised weight is the product of
    the normalised 1-D weights; all factors are powers of two, so the values
    are bit-identical to the reference's.
    """
    wx, wy, wz = (_weights_1d(f, c) for f, c in zip(fine, coarse))
    nyf, nzf = fine[1] + 1, fine[2] + 1
    nyc, nzc = coarse[1] + 1, coarse[2] + 1
    rows, cols, vals = [], [], []
    for i, px in enumerate(wx):
        for j, py in enumerate(wy):
            for k, pz in enumerate(wz):
                r = (i * nyf + j) * nzf + k
                for ci, a in px:
                    for cj, b in py:
                        for ck, c in pz:
                            rows.append(r)
                            cols.append((ci * nyc + cj) * nzc + ck)
                            vals.append(a * b * c)
    nf = (fine[0] + 1) * nyf * nzf
    nc = (coarse[0] + 1) * nyc * nzc
    return sp.csr_matrix((vals, (rows, cols)), shape=(nf, nc))


def injection_free(fine, coarse, free_f) -> np.ndarray:
    """Coarse free DoFs by injection (solver_v2.py:717-764): coarse node
    (I,J,K) is free in component d iff fine node (2I,2J,2K) is."""
    nd_f = fem.n_dof(fine)
    mask_f = np.zeros(nd_f, dtype=bool)
    mask_f[free_f] = True
    I, J, K = np.meshgrid(*(np.arange(c + 1) for c in coarse), indexing="ij")
    fn = ((2 * I * (fine[1] + 1) + 2 * J) * (fine[2] + 1) + 2 * K).ravel()
    is_free = np.zeros(fem.n_dof(coarse), dtype=bool)
    for d in range(3):
        fd = 3 * fn + d
        ok = fd < nd_f
        is_free[(3 * np.arange(len(fn)) + d)[ok]] = mask_f[fd[ok]]
    return np.nonzero(is_free)[0].astype(np.int64)


def local_prolongation(s: int, t: int, u: int) -> np.ndarray:
    """8x8 weights from a coarse hex's corners to the corners of its fine
    sub-hex (s,t,u) (multigrid_v4.py:105-129)."""
    P = np.zeros((8, 8))
    for fn in range(8):
        x = (np.array([s, t, u]) + fem.CORNERS[fn]) / 2.0
        for cn in range(8):
            w = 1.0
            for d in range(3):
                w *= x[d] if fem.CORNERS[cn][d] else 1.0 - x[d]
            P[fn, cn] = w
    return P


def galerkin_blocks(KE: np.ndarray = fem.KE_UNIT) -> np.ndarray:
    """Q_stu = P24^T KE P24 for the 8 sub-hexes, order s-major (multigrid_v4.py:182-187)."""
    Q = []
    for s in range(2):
        for t in range(2):
            for u in range(2):
                P24 = np.kron(local_prolongation(s, t, u), np.eye(3))
                Q.append(P24.T @ KE @ P24)
    return np.stack(Q)


def level1_galerkin(E_f, fine, coarse, free_c, KE: np.ndarray = fem.KE_UNIT) -> sp.csr_matrix:
    """Level-1 operator from coarse element matrices sum_stu E_f Q_stu with the
    fine element index clamped to the fine grid (multigrid_v4.py:132-270),
    restricted to free_c x free_c."""
    Q = galerkin_blocks(KE)
    nxc, nyc, nzc = coarse
    cx, cy, cz = np.meshgrid(np.arange(nxc), np.arange(nyc), np.arange(nzc), indexing="ij")
    cx, cy, cz = cx.ravel(), cy.ravel(), cz.ravel()
    Kc = np.zeros((len(cx), 24, 24))
    q = 0
    for s in range(2):
        for t in range(2):
            for u in range(2):
                fx = np.minimum(2 * cx + s, fine[0] - 1)
                fy = np.minimum(2 * cy + t, fine[1] - 1)
                fz = np.minimum(2 * cz + u, fine[2] - 1)
                Ef = np.asarray(E_f)[(fx * fine[1] + fy) * fine[2] + fz]
                Kc += Ef[:, None, None] * Q[q][None]
                q += 1
    edof = fem.edof_table(coarse).astype(np.int64)
    rows = np.repeat(edof, 24, axis=1).ravel()
    cols = np.tile(edof, (1, 24)).ravel()
    nd = fem.n_dof(coarse)
    K = sp.csr_matrix((Kc.ravel(), (rows, cols)), shape=(nd, nd))
    return K[free_c][:, free_c].tocsr()


def _guard_diag(d):
    """Zero-guard used for every Jacobi diagonal (multigrid_v4.py:269,685,752)."""
    return np.where(np.abs(d) > 1e-12, d, 1.0)


def lambda_fine(matvec, d_inv, n_iter: int = 20) -> float:
    """D-norm power iteration for lambda_max(D^-1 K) (multigrid_v4.py:273-295)."""
    d = 1.0 / d_inv
    v = np.ones(len(d_inv))
    v /= np.sqrt(np.dot(v * d, v))
    lam = 1.0
    for _ in range(n_iter):
        Kv = matvec(v)
        lam = np.dot(v, Kv) / max(np.dot(v * d, v), 1e-300)
        Av = d_inv * Kv
        nrm = np.sqrt(np.dot(Av * d, Av))
        if nrm <= 1e-300:
            break
        v = Av / nrm
    return float(lam)


def lambda_sparse(K, d_inv, n_iter: int = 10) -> float:
    """Power iteration at a coarse level (multigrid_v4.py:298-314)."""
    v = np.ones(len(d_inv))
    v /= np.linalg.norm(v)
    lam = 1.0
    for _ in range(n_iter):
        Kv = K @ v
        Av = d_inv * Kv
        nrm = np.linalg.norm(Av)
        if nrm <= 1e-300:
            break
        lam = np.dot(v, Kv) / max(np.dot(v, v / d_inv), 1e-300)
        v = Av / nrm
    return max(float(lam), 1e-6)


def chebyshev(A, rhs, x0, d_inv, lam_max, lower_frac, degree, x0_is_zero=False):
    """Chebyshev-Jacobi smoothing, Saad Alg. 12.1 (multigrid_v4.py:861-889).

    Works for any array dtype; scalars follow the dtype of ``rhs``. With
    ``x0_is_zero`` the first residual is ``rhs`` itself (A.0 = 0 exactly).
    """
    dt = rhs.dtype.type
    lam_max = dt(lam_max)
    lam_min = dt(lower_frac) * lam_max
    sigma = (lam_max + lam_min) * dt(0.5)
    delta = (lam_max - lam_min) * dt(0.5)
    x = x0
    r = rhs if x0_is_zero else rhs - A(x)
    alpha = dt(2.0) / (lam_max + lam_min)
    d = d_inv * r
    x = x + alpha * d
    for _ in range(1, degree):
        r = rhs - A(x)
        z = d_inv * r
        alpha_new = dt(1.0) / (sigma - delta**2 * alpha * dt(0.25))
        d = alpha_new * (z + delta**2 * alpha * dt(0.25) * d)
        x = x + d
        alpha = alpha_new
    return x


def fixed_pcg(K, b, d_inv, n_iters: int = 80):
    """Fixed-count Jacobi-PCG for the coarsest level (solver_v2.py:782-811)."""
    x = np.zeros_like(b)
    r = b.copy()
    z = d_inv * r
    p = z.copy()
    rz = r.dot(z)
    for _ in range(n_iters):
        Ap = K @ p
        alpha = rz / (p.dot(Ap) + 1e-300)
        x = x + alpha * p
        r = r - alpha * Ap
        z = d_inv * r
        rz_n = r.dot(z)
        beta = rz_n / (rz + 1e-300)
        p = z + beta * p
        rz = rz_n
    return x


class GMG:
    """Restatement of GalerkinMatFreeGMG with the SolverV4 defaults.

    ``fine_prec`` selects the fine-smoother arithmetic ("fp64", "fp32" or
    "bf16"); coarse levels follow the reference's default schedule
    (multigrid_v4.py:673-682) unless ``level_prec`` is given.
    """

    def __init__(self, nel, free, n_levels=4, fine_prec="fp64", fine_degree=2, coarse_iters=2,
                 cheb_lower_frac=1.0 / 30.0, dense_chol_max=5000, coarse_pcg_iters=80,
                 level_prec=None, cycle="v"):
        if cycle not in ("v", "w"):
            raise ValueError("cycle must be 'v' or 'w'")
        self.cycle = cycle
        self.nel = tuple(nel)
        self.n_levels = n_levels
        self.fine_prec = fine_prec
        self.fine_degree = max(1, fine_degree)
        self.coarse_iters = max(1, coarse_iters)
        self.lower = cheb_lower_frac
        self.dense_chol_max = dense_chol_max
        self.coarse_pcg_iters = coarse_pcg_iters
        self.dims = level_dims(nel, n_levels)
        self.free = [np.asarray(free, dtype=np.int64)]
        self.P = []
        for lv in range(n_levels - 1):
            fc = injection_free(self.dims[lv], self.dims[lv + 1], self.free[lv])
            Ps = scalar_prolongation(self.dims[lv], self.dims[lv + 1])
            Pv = sp.kron(Ps, sp.eye(3), format="csr")
            self.P.append(Pv[self.free[lv], :][:, fc].tocsr())
            self.free.append(fc)
        if level_prec is None:
            if fine_prec == "bf16":
                level_prec = ["bf16"] + (["fp32"] if n_levels > 1 else [])
            else:
                level_prec = [fine_prec]
        self.level_prec = list(level_prec) + ["fp64"] * (n_levels - len(level_prec))
        self.lam = [np.nan] * n_levels
        self._lam_Emax = np.nan

    # -- setup (multigrid_v4.py:657-813) ---------------------------------
    def setup(self, E):
        self.E = np.asarray(E, dtype=np.float64)
        nd = fem.n_dof(self.nel)
        f0 = self.free[0]
        d0 = fem.diagonal_full(self.E, self.nel)[f0]
        self.d_inv = [1.0 / _guard_diag(d0)]
        Emax = float(self.E.max())
        re = np.isnan(self._lam_Emax) or abs(Emax - self._lam_Emax) / max(abs(self._lam_Emax), 1e-12) > 0.10
        if re:
            self.lam[0] = lambda_fine(self.fine_op64, self.d_inv[0])
            self._lam_Emax = Emax
        self.K = [None]
        if self.n_levels > 1:
            K1 = level1_galerkin(self.E, self.dims[0], self.dims[1], self.free[1])
            self.K.append(K1)
            self.d_inv.append(1.0 / _guard_diag(K1.diagonal()))
            if re or np.isnan(self.lam[1]):
                self.lam[1] = lambda_sparse(K1, self.d_inv[1])
        for lv in range(2, self.n_levels):
            Kc = (self.P[lv - 1].T @ (self.K[lv - 1] @ self.P[lv - 1])).tocsr()
            Kc.sum_duplicates()
            self.K.append(Kc)
            self.d_inv.append(1.0 / _guard_diag(Kc.diagonal()))
            if re or np.isnan(self.lam[lv]):
                self.lam[lv] = lambda_sparse(Kc, self.d_inv[lv])
        self.chol = None
        if self.n_levels > 1:
            Kd = self.K[-1].toarray()
            if Kd.shape[0] <= self.dense_chol_max:
                try:
                    L = np.linalg.cholesky(Kd)
                    if not np.all(np.isfinite(L)):
                        raise np.linalg.LinAlgError
                    self.chol = L
                except np.linalg.LinAlgError:
                    eps = max(float(Kd.diagonal().mean()) * 1e-8, 1e-14)
                    try:
                        self.chol = np.linalg.cholesky(Kd + eps * np.eye(Kd.shape[0]))
                    except np.linalg.LinAlgError:
                        self.chol = None
        _ = nd
        return self

    def fine_op64(self, v):
        return fem.matvec_free(v, self.E, self.nel, self.free[0], "fp64")

    def _fine_op_low(self, v):
        return fem.matvec_free(v, self.E.astype(np.float32), self.nel, self.free[0], self.level_prec[0])

    def smooth_fine(self, x, rhs, x_is_zero=False):
        prec = self.level_prec[0]
        if prec == "fp64":
            return chebyshev(self.fine_op64, rhs, x.copy(), self.d_inv[0], self.lam[0], self.lower,
                             self.fine_degree, x_is_zero)
        x32 = chebyshev(self._fine_op_low, rhs.astype(np.float32), x.astype(np.float32),
                        self.d_inv[0].astype(np.float32), np.float32(self.lam[0]), np.float32(self.lower),
                        self.fine_degree, x_is_zero)
        return x32.astype(np.float64)

    def smooth_coarse(self, lv, x, rhs, x_is_zero=False):
        lam = self.lam[lv] if np.isfinite(self.lam[lv]) else 1.0
        if self.level_prec[lv] in ("fp32", "bf16"):
            K32 = self.K[lv].astype(np.float32)
            x32 = chebyshev(lambda v: K32 @ v, rhs.astype(np.float32), x.astype(np.float32),
                            self.d_inv[lv].astype(np.float32), np.float32(lam), np.float32(self.lower),
                            self.coarse_iters, x_is_zero)
            return x32.astype(np.float64)
        K = self.K[lv]
        return chebyshev(lambda v: K @ v, rhs, x, self.d_inv[lv], lam, self.lower, self.coarse_iters, x_is_zero)

    def solve_coarsest(self, rhs):
        lv = self.n_levels - 1
        if self.chol is not None:
            y = sla.solve_triangular(self.chol, rhs, lower=True)
            return sla.solve_triangular(self.chol, y, lower=True, trans="T")
        return fixed_pcg(self.K[lv], rhs, self.d_inv[lv], self.coarse_pcg_iters)

    def vcycle(self, lv, rhs):
        """multigrid_v4.py:986-1008."""
        if lv == self.n_levels - 1:
            if self.n_levels == 1:
                return self.smooth_fine(np.zeros_like(rhs), rhs, True)
            return self.solve_coarsest(rhs)
        z = np.zeros_like(rhs)
        if lv == 0:
            x = self.smooth_fine(z, rhs, True)
            res = rhs - self.fine_op64(x)
        else:
            x = self.smooth_coarse(lv, z, rhs, True)
            res = rhs - self.K[lv] @ x
        ec = self.vcycle(lv + 1, self.P[lv].T @ res)
        x = x + self.P[lv] @ ec
        return self.smooth_fine(x, rhs) if lv == 0 else self.smooth_coarse(lv, x, rhs)

    def wcycle(self, lv, rhs):
        """multigrid_v4.py:1010-1042: two coarse corrections per level, the
        second on the residual after the first."""
        if lv == self.n_levels - 1:
            if self.n_levels == 1:
                return self.smooth_fine(np.zeros_like(rhs), rhs, True)
            return self.solve_coarsest(rhs)
        z = np.zeros_like(rhs)
        op = self.fine_op64 if lv == 0 else (lambda v: self.K[lv] @ v)
        x = self.smooth_fine(z, rhs, True) if lv == 0 else self.smooth_coarse(lv, z, rhs, True)
        x = x + self.P[lv] @ self.wcycle(lv + 1, self.P[lv].T @ (rhs - op(x)))
        x = x + self.P[lv] @ self.wcycle(lv + 1, self.P[lv].T @ (rhs - op(x)))
        return self.smooth_fine(x, rhs) if lv == 0 else self.smooth_coarse(lv, x, rhs)

    def apply(self, r):
        r = np.asarray(r, dtype=np.float64)
        return self.wcycle(0, r) if self.cycle == "w" else self.vcycle(0, r)
