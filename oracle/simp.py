"""Oracle: SolverV4 state solve and SIMP loops (TEST INFRASTRUCTURE)."""

from __future__ import annotations

import numpy as np

from . import design, fem, gmg, krylov


class StateSolverV4:
    """Restates ``SolverV4._solve_cupy_matfree`` (solver_v4.py:147-269) with
    the settings ``SIMPSolver(backend="cuda")`` passes (topogpu/solver.py:199-219):
    matrix-free FP64 outer operator, Galerkin GMG preconditioner, PCG (or
    FGMRES for a BF16 smoother), warm start with the reset rule of
    solver_v4.py:162-165 and the cold retry of solver_v4.py:201-209."""

    def __init__(self, nel, bc: fem.BC, n_levels=4, fine_prec="fp64", fine_degree=2, tol=1e-5,
                 maxiter=800, outer="auto", E0=1.0, Emin=1e-9, **gmg_kw):
        self.nel = tuple(nel)
        self.bc = bc
        self.tol, self.maxiter = tol, maxiter
        self.E0, self.Emin = E0, Emin
        self.gmg = gmg.GMG(nel, bc.free, n_levels=n_levels, fine_prec=fine_prec,
                           fine_degree=fine_degree, **gmg_kw)
        self.outer = ("fgmres" if fine_prec == "bf16" else "pcg") if outer == "auto" else outer
        self.u_prev = None
        self.prev_penal = None
        self.last_iters = 0
        self.last_u_full = None

    def solve(self, rho, penal=3.0):
        if self.prev_penal is not None and abs(penal - self.prev_penal) > 0.5:
            self.u_prev = None
        self.prev_penal = penal
        rho = np.asarray(rho, dtype=np.float64)
        E = self.Emin + (self.E0 - self.Emin) * rho**penal
        self.gmg.setup(E)
        F = self.bc.F[self.bc.free]
        A = self.gmg.fine_op64
        solver = krylov.pcg if self.outer == "pcg" else krylov.fgmres
        u, it, ok = solver(A, F, self.gmg.apply, x0=self.u_prev, tol=self.tol, maxiter=self.maxiter)
        if not ok and self.u_prev is not None:
            u, it, ok = solver(A, F, self.gmg.apply, x0=None, tol=self.tol, maxiter=self.maxiter)
        self.last_iters, self.converged = it, ok
        self.u_prev = u.copy()
        compliance = float(np.dot(F, u))
        U = np.zeros(self.bc.ndof)
        U[self.bc.free] = u
        self.last_u_full = U
        dc = fem.sensitivity(U, rho, self.nel, penal, self.E0, self.Emin)
        return compliance, dc


def simp_solverv4(nel, bc, volfrac, max_iter, move=0.10, rho_min=1e-3, **kw):
    """SIMPSolver._solve_solverv4 loop (topogpu/solver.py:186-249): no filter,
    OC on the plain mean. Returns (rho, compliance history, per-iteration rho)."""
    st = StateSolverV4(nel, bc, **kw)
    rho = np.full(int(np.prod(nel)), float(volfrac))
    comp, rhos = [], []
    for _ in range(max_iter):
        c, dc = st.solve(rho, 3.0)
        rho, _ = design.oc_update(rho, dc, volfrac, move, rho_min)
        comp.append(c)
        rhos.append(rho.copy())
    return rho, comp, rhos


class FilteredSIMP:
    """run_simp-style filtered SIMP whose state solve is the SolverV4 GMG-PCG
    restatement (the reference's GPU algorithm run on the host): one
    ``step()`` = filter, state solve, sensitivity, H^T chain, filtered OC.
    Used as the timed CPU baseline."""

    def __init__(self, nel, bc, volfrac, rmin, move=0.2, penal=3.0, **solver_kw):
        self.nel, self.bc = tuple(nel), bc
        self.H = design.filter_matrix(nel, rmin)
        n = self.H.shape[0]
        self.rho = np.full(n, float(volfrac))
        self.dv = self.H.T @ np.ones(n)
        self.volfrac, self.move, self.penal = volfrac, move, penal
        self.state = StateSolverV4(nel, bc, **solver_kw)

    def step(self):
        rp = self.H @ self.rho
        c, dc = self.state.solve(rp, self.penal)
        self.rho, _ = design.oc_update_filtered(self.rho, self.H.T @ dc, self.dv, self.volfrac, self.move, self.H)
        return c


def simp_projected(nel, bc, volfrac, rmin, max_iter, beta, eta=0.5, move=0.2, penal=3.0):
    """``run_simp`` main loop with Heaviside projection at a fixed beta
    (_fea_and_sensitivity, pub_simp_solver.py:342-377): rho_phys =
    heaviside(H rho), direct solve, dc chained through dh and H^T, dv = H^T dh,
    OC with the projected volume. Returns (rho_design, compliance history,
    final compliance, final rho_phys) like ``simp_filtered``."""
    H = design.filter_matrix(nel, rmin)
    n = H.shape[0]
    rho = np.full(n, float(volfrac))
    hist = []

    def fea(r):
        rf = H @ r
        rp = design.heaviside(rf, beta, eta)
        E = 1e-9 + (1.0 - 1e-9) * rp**penal
        U = fem.direct_solve(E, nel, bc)
        dcp = -penal * (1.0 - 1e-9) * rp ** (penal - 1) * fem.element_energy(U, nel)
        dh = design.heaviside_deriv(rf, beta, eta)
        return float(bc.F @ U), rp, H.T @ (dcp * dh), H.T @ dh

    for _ in range(max_iter):
        c, rp, dcd, dvd = fea(rho)
        hist.append(c)
        rho, _ = design.oc_update_projected(rho, dcd, dvd, volfrac, move, H, beta, eta)
    cf, rpf, _, _ = fea(rho)
    return rho, hist, cf, rpf


def simp_filtered(nel, bc, volfrac, rmin, max_iter, move=0.2, penal=3.0, solve=None):
    """``run_simp`` main loop without Heaviside, callbacks or tail
    (pub_simp_solver.py:412-657, _fea_and_sensitivity 342-377): physical
    density H*rho, direct solve, sensitivity chained through H^T, filtered-
    volume OC. ``solve(E)`` may replace the direct solve. Returns
    (rho_design, compliance history, final compliance, final rho_phys)."""
    H = design.filter_matrix(nel, rmin)
    n = H.shape[0]
    rho = np.full(n, float(volfrac))
    dv = H.T @ np.ones(n)
    hist = []

    def fea(r):
        rp = H @ r
        E = 1e-9 + (1.0 - 1e-9) * rp**penal
        U = fem.direct_solve(E, nel, bc) if solve is None else solve(E)
        c = float(bc.F @ U)
        dcp = -penal * (1.0 - 1e-9) * rp ** (penal - 1) * fem.element_energy(U, nel)
        return c, rp, H.T @ dcp

    for _ in range(max_iter):
        c, rp, dcd = fea(rho)
        hist.append(c)
        rho, _ = design.oc_update_filtered(rho, dcd, dv, volfrac, move, H)
    cf, rpf, _ = fea(rho)
    return rho, hist, cf, rpf
