"""State solve of one SIMP iteration on the device (SolverV4 equivalent).

``StateSolver.solve(rho, penal) -> (compliance, dc)`` keeps the contract of
the reference's ``SolverV4.solve`` (src/gpu_fem/solver_v4.py:147-269): E(rho),
GMG setup, warm-started Krylov solve with a cold retry when it fails, the
compliance F.u and the element-energy sensitivity. Everything runs in
libtopo_b200.so; rho and dc are CUDA tensors (NumPy input is uploaded).
"""

from __future__ import annotations

import numpy as np
import torch

from .context import TopoContext


class StateSolver:
    """Matrix-free GMG-preconditioned state solve on a structured hex8 grid.

    Parameters mirror SolverV4's (solver_v4.py:38-89): ``n_levels``
    (matfree_gmg_levels), ``fine_degree`` (gmg_fine_degree), ``coarse_degree``
    (gmg_smooth_iters), ``cheb_lower`` (gmg_cheb_lower_frac), ``outer``
    ("pcg" or "fgmres"), ``tol``/``maxiter`` (cg_tol/cg_maxiter),
    ``warm_start``. ``precision`` selects the arithmetic schedule
    ("fp64", "fp32" or "mixed", see include/topo_b200.h); ``smoother`` is
    "chebyshev" (default) or "reference" (the reference V-cycle exactly).
    """

    def __init__(self, nel, free_mask, F, *, n_levels=4, precision="mixed", fine_degree=2, coarse_degree=2,
                 cheb_lower=1.0 / 30.0, outer="pcg", restart=32, tol=1e-5, maxiter=800, warm_start=True,
                 E0=1.0, Emin=1e-9, dense_max=16384, smoother="chebyshev", probe=False, cycle_type="v",
                 KE=None, device=None):
        if outer not in ("pcg", "fgmres"):
            raise ValueError(f"outer must be 'pcg' or 'fgmres', got {outer!r}")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        with torch.cuda.device(self.device):
            self.ctx = TopoContext(nel, n_levels=n_levels, mode=precision, fine_degree=fine_degree,
                                   coarse_degree=coarse_degree, cheb_lower=cheb_lower, dense_max=dense_max,
                                   KE=KE, smoother=smoother)
        self.ctx.set_cycle(cycle_type)
        self.cycle_type = cycle_type
        self.nel = self.ctx.nel
        self.precision = precision
        self.outer, self.restart = outer, restart
        self.tol, self.maxiter = tol, maxiter
        self.warm_start = warm_start
        self.E0, self.Emin = E0, Emin
        dev = self.device
        self.free_mask = torch.as_tensor(np.asarray(free_mask, dtype=np.uint8), device=dev).contiguous()
        self.F = torch.as_tensor(np.asarray(F, dtype=np.float64), device=dev).contiguous()
        self.ctx.set_problem(self.free_mask, self.F)
        self.b = (self.F * self.free_mask).contiguous()
        self.u = torch.zeros(self.ctx.ndof, dtype=torch.float64, device=dev)
        self.E = torch.empty(self.ctx.n_elem, dtype=torch.float64, device=dev)
        self._have_prev = False
        self._prev_penal = None
        self.last_cg_iters = 0
        self.last_relres = float("nan")
        self.last_converged = False
        self.last_outer_solver = outer
        self.last_timing: dict = {}
        self.probe = probe  # one extra V-cycle per solve for last_multigrid_quality
        self.last_multigrid_quality: dict = {}

    def _krylov(self):
        if self.outer == "pcg":
            return self.ctx.pcg(self.b, self.u, self.tol, self.maxiter)
        return self.ctx.fgmres(self.b, self.u, self.tol, self.maxiter, self.restart)

    timing = False  # set True to fill last_timing on every solve (adds one sync)

    def solve(self, rho, penal: float = 3.0, *, timing: bool = False):
        dev = self.device
        timing = timing or self.timing
        rho = torch.as_tensor(rho, dtype=torch.float64, device=dev).contiguous()
        if self._prev_penal is not None and abs(penal - self._prev_penal) > 0.5:
            self._have_prev = False
        self._prev_penal = penal
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)] if timing else None
        if timing:
            ev[0].record()
        self.ctx.modulus(rho, penal, self.E0, self.Emin, out=self.E)
        self.ctx.gmg_setup(self.E)
        if timing:
            ev[1].record()
        if self.probe:
            self.last_multigrid_quality = self.probe_quality()
        warm = self.warm_start and self._have_prev
        if not warm:
            self.u.zero_()
        it, rr, ok = self._krylov()
        if not ok and warm:
            self.u.zero_()
            it, rr, ok = self._krylov()
        if timing:
            ev[2].record()
        self.last_cg_iters, self.last_relres, self.last_converged = it, rr, ok
        self._have_prev = True
        compliance = self.ctx.dot(self.F, self.u)
        dc = self.ctx.sensitivity(self.u, rho, penal, self.E0, self.Emin)
        if timing:
            ev[3].record()
            torch.cuda.synchronize(dev)
            self.last_timing = {"gmg_setup_ms": ev[0].elapsed_time(ev[1]), "cg_ms": ev[1].elapsed_time(ev[2]),
                                "sensitivity_ms": ev[2].elapsed_time(ev[3]), "total_ms": ev[0].elapsed_time(ev[3]),
                                "outer_solver": self.outer, "cg_iters": it}
        return float(compliance), dc

    def solve_block(self, rho, loads, penal: float = 3.0):
        """Several load cases on one density field with block PCG.

        loads: (nrhs, ndof) float64 (fixed DoFs ignored). Returns
        (compliances F_j . u_j as a list, U as an (nrhs, ndof) tensor). The
        hierarchy is set up once for all load cases."""
        dev = self.device
        rho = torch.as_tensor(rho, dtype=torch.float64, device=dev).contiguous()
        B = torch.as_tensor(loads, dtype=torch.float64, device=dev).contiguous()
        self.ctx.modulus(rho, penal, self.E0, self.Emin, out=self.E)
        self.ctx.gmg_setup(self.E)
        U = torch.zeros_like(B)
        it, rr, ok = self.ctx.block_pcg(B, U, self.tol, self.maxiter)
        self.last_cg_iters, self.last_relres, self.last_converged = it, max(rr), ok
        self.last_outer_solver = "block_pcg"
        Bm = B * self.free_mask
        return [float(torch.dot(Bm[j], U[j])) for j in range(B.shape[0])], U

    # -- diagnostics (GalerkinMatFreeGMG.probe_quality / estimate_kappa_eff) --
    def _precondition(self, r):
        vdt = self.ctx.vec_dtype
        return self.ctx.gmg_apply(r.to(vdt).contiguous()).to(torch.float64)

    def probe_quality(self, rhs=None) -> dict:
        """One V-cycle on rhs (default: the load) with the current hierarchy:
        finiteness, positivity of rhs.z and the norms of z and of the Jacobi
        step, as GalerkinMatFreeGMG.probe_quality (multigrid_v4.py:821-832)."""
        rhs = (self.F * self.free_mask) if rhs is None else rhs.to(torch.float64) * self.free_mask
        z = self._precondition(rhs)
        d = self.ctx.diag(self.E)
        zj = torch.where(self.free_mask.bool(), rhs / d, torch.zeros_like(rhs))
        return {"finite": bool(torch.isfinite(z).all()), "pd": float(torch.dot(rhs, z)) > 0.0,
                "z_norm": float(z.norm()), "jacobi_norm": float(zj.norm())}

    def estimate_kappa_eff(self, n_iter: int = 30, seed: int = 0) -> float:
        """lambda_max / lambda_min of the n_iter-step Lanczos tridiagonal of the
        preconditioned operator M K on the current hierarchy (Euclidean inner
        product, seeded normal start vector), as
        GalerkinMatFreeGMG.estimate_kappa_eff (multigrid_v4.py:606-655)."""
        g = torch.Generator().manual_seed(seed)
        m = self.free_mask.to(torch.float64)
        v = torch.randn(self.ctx.ndof, generator=g, dtype=torch.float64).to(self.device) * m
        v /= v.norm()
        v_prev = torch.zeros_like(v)
        alphas, betas = [], []
        for j in range(n_iter):
            w = self._precondition(self.ctx.matvec(v, self.E))
            a = float(torch.dot(v, w))
            alphas.append(a)
            w = w - a * v
            if j > 0:
                w = w - betas[-1] * v_prev
            if j < n_iter - 1:
                b = float(w.norm())
                if b < 1e-14:
                    break
                betas.append(b)
                v_prev, v = v, w / b
        betas = betas[: len(alphas) - 1]
        T = np.diag(alphas) + np.diag(betas, 1) + np.diag(betas, -1)
        eig = np.linalg.eigvalsh(T)
        eig = eig[eig > 0]
        self.last_kappa_eff = float(eig[-1] / max(eig[0], 1e-300)) if len(eig) else float("nan")
        return self.last_kappa_eff

    def reset_warm_start(self):
        """Make the next solve start from u = 0."""
        self._have_prev = False

    def displacement(self) -> torch.Tensor:
        """Last displacement (full length, fixed DoFs zero) in FP64."""
        return self.u

    def close(self):
        self.ctx.close()
