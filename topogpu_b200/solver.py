"""Public SIMP driver: ``SIMPSolver(backend="cuda", ...).solve(problem)``.

Drop-in for the reference's SolverV4 path (src/topogpu/solver.py:124-253):
same constructor arguments, same ``OptimizationResult`` and evidence bundle,
same history/summary keys. Each iteration runs entirely on the GPU: E(rho),
GMG setup, Krylov solve, compliance, sensitivity and the bisection OC update
(the reference does the OC in host NumPy); the host only reads the scalars
that go into the history rows.

Defaults reproduce the reference path: no density filter, penalty 3,
OC on the plain mean volume. ``backend="cpu"`` (the default, as in the
reference: its CPU backend, ``run_simp``) runs that driver with its physics
on the GPU (``topogpu_b200.run_simp``). ``use_filter=True`` switches to the filtered
formulation of the reference's CPU driver ``run_simp``
(src/gpu_fem/pub_simp_solver.py:342-377): physical density H rho,
sensitivities chained through H^T, volume measured after the filter.
``use_heaviside=True`` (with ``use_filter``) adds run_simp's smoothed
Heaviside projection at ``beta``/``eta`` (pub_simp_solver.py:245-253,
342-377): rho_phys = h(H rho), sensitivities chained through h' and H^T, the
OC volume measured after filter and projection. ``SIMPLoop.beta`` may be
changed between steps (run_simp's continuation changes beta the same way,
between iterations, 379-386).
"""

from __future__ import annotations

import os
import time
from dataclasses import dataclass
from pathlib import Path
from typing import Any

import numpy as np
import torch

from .bc import generate_bc
from .checkpoint import checkpoint_path, load_checkpoint, save_checkpoint
from .evidence import EvidenceBundle
from .problem import TopologyProblem
from .state import StateSolver


@dataclass
class SIMPModel:
    penal: float = 3.0
    rho_min: float = 1.0e-3


@dataclass
class OCOptimizer:
    move: float = 0.10


@dataclass
class OptimizationResult:
    problem: TopologyProblem
    rho_final: np.ndarray
    history: list
    summary: dict

    def save(self, path) -> EvidenceBundle:
        bundle = EvidenceBundle(Path(path))
        bundle.write_history(self.history)
        bundle.write_density(self.rho_final)
        bundle.write_render_metadata({"density_threshold": 0.5, "scalar": "density",
                                      "scalar_normalization": "per_case_0_1", "camera": "orthographic_default",
                                      "source": "OptimizationResult.save"})
        bundle.write_summary(self.summary)
        bundle.write_manifest()
        return bundle


_PRECISIONS = ("fp64", "fp32", "mixed")


class SIMPSolver:
    """Bounded SIMP loop on one B200.

    Reference arguments: backend, linear_solver, optimizer, tol, max_krylov,
    max_iter, move, rho_min. Extra (optional) arguments: precision
    ("mixed" default, "fp32", "fp64"), levels, fine_degree, coarse_degree,
    use_filter, use_heaviside, beta, eta, penal, smoother ("chebyshev"
    default, "reference"), checkpoint_dir / checkpoint_every /
    checkpoint_problem (run_simp's checkpoint files: resume from one when it
    exists, write one every checkpoint_every iterations), cycle_type ("v"
    default, "w": SolverV4's gmg_cycle_type), device.
    """

    def __init__(self, backend="cpu", linear_solver="auto", optimizer="oc", tol=1.0e-5, max_krylov=800,
                 max_iter=12, move=0.10, rho_min=1.0e-3, *, precision="mixed", levels=4, fine_degree=2,
                 coarse_degree=2, use_filter=False, use_heaviside=False, beta=1.0, eta=0.5, penal=3.0,
                 smoother="chebyshev", coarse_lag=None, checkpoint_dir=None, checkpoint_every=10,
                 checkpoint_problem="cantilever", cycle_type="v", device=None):
        if optimizer != "oc":
            raise ValueError("Only optimizer='oc' is implemented in v0.1.0.")
        if backend not in {"cuda", "cupy", "cpu", "scipy"}:
            raise ValueError(f"Unknown backend {backend!r}.")
        if linear_solver not in {"auto", "pcg_gmg", "fgmres_gmg"}:
            raise ValueError(f"Unknown linear_solver {linear_solver!r}.")
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {_PRECISIONS}, got {precision!r}")
        self.backend = backend
        self.linear_solver = linear_solver
        self.tol, self.max_krylov, self.max_iter = tol, max_krylov, max_iter
        self.move, self.rho_min = move, rho_min
        self.precision, self.levels = precision, levels
        self.fine_degree, self.coarse_degree = fine_degree, coarse_degree
        if use_heaviside and not use_filter:
            raise ValueError("use_heaviside=True needs use_filter=True (run_simp projects the filtered density)")
        self.use_filter = use_filter
        self.use_heaviside = bool(use_heaviside)
        self.beta, self.eta = float(beta), float(eta)
        self.penal = penal
        self.smoother = smoother
        # one-setup-lagged coarsest factor built in the background: off by default
        # (on the 1M-element SIMP run it saved the factorisation time but cost as
        # much in extra PCG iterations and in contention with the Krylov kernels)
        self.coarse_lag = bool(coarse_lag) if coarse_lag is not None else False
        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be >= 1")
        self.checkpoint_dir, self.checkpoint_every = checkpoint_dir, int(checkpoint_every)
        self.checkpoint_problem = checkpoint_problem
        if cycle_type not in ("v", "w"):
            raise ValueError(f"cycle_type must be 'v' or 'w'; got {cycle_type!r}")
        self.cycle_type = cycle_type
        self.device = device

    def make_state_solver(self, problem: TopologyProblem) -> StateSolver:
        spec = problem.spec
        if not problem.is_3d:
            raise ValueError("SolverV4 backend currently requires a 3D problem.")
        bc = generate_bc(spec)
        F = problem.force_override if problem.force_override is not None else bc.F
        outer = "fgmres" if self.linear_solver == "fgmres_gmg" else "pcg"
        st = StateSolver(problem.nel, bc.free_mask(), F, n_levels=self.levels, precision=self.precision,
                         fine_degree=self.fine_degree, coarse_degree=self.coarse_degree, outer=outer,
                         tol=self.tol, maxiter=self.max_krylov, smoother=self.smoother, cycle_type=self.cycle_type,
                         device=self.device)
        st.ctx.set_coarse_lag(self.coarse_lag)
        return st

    def solve(self, problem: TopologyProblem) -> OptimizationResult:
        problem.validate()
        if self.backend in {"cpu", "scipy"}:
            return self._solve_run_simp(problem)
        loop = SIMPLoop(self, problem, track_best=self.checkpoint_dir is not None)
        try:
            ckpt_path = None
            if self.checkpoint_dir is not None:
                os.makedirs(self.checkpoint_dir, exist_ok=True)
                ckpt_path = checkpoint_path(self.checkpoint_dir, problem.nel, self.checkpoint_problem)
                ck = load_checkpoint(ckpt_path)
                if ck is not None:
                    loop.restore(ck)
            history: list[dict[str, Any]] = []
            t_total = time.perf_counter()
            while loop.iteration < self.max_iter:
                t0 = time.perf_counter()
                row = loop.step()
                row["wall_s"] = time.perf_counter() - t0
                history.append(row)
                if ckpt_path is not None and loop.iteration % self.checkpoint_every == 0:
                    loop.save_checkpoint(ckpt_path)
            summary = {"problem": problem.to_dict(), "backend": "SolverV4-B200",
                       "linear_solver": "pcg_gmg" if self.linear_solver == "auto" else self.linear_solver,
                       "precision": self.precision, "n_iter": len(history),
                       "total_wall_s": time.perf_counter() - t_total, "final": history[-1] if history else {}}
            return OptimizationResult(problem, loop.rho.cpu().numpy(), history, summary)
        finally:
            loop.close()


    def _solve_run_simp(self, problem: TopologyProblem) -> OptimizationResult:
        """The reference's ``backend="cpu"`` path (src/topogpu/solver.py:156-184):
        ``run_simp`` with the same parameters (radius, move, tol 1e-3,
        min_iter min(2, max_iter), Heaviside at beta 1), here with its physics
        on the GPU. The problem's own supports and loads are used; the
        reference drops them there and solves run_simp's tip-load preset."""
        from .run_simp import SIMPParams, run_simp

        spec = problem.spec
        if not problem.is_3d:
            raise ValueError("the B200 run_simp path handles 3-D problems only")
        bc = generate_bc(spec)
        F = problem.force_override if problem.force_override is not None else bc.F
        params = SIMPParams(nelx=spec.nelx, nely=spec.nely, nelz=spec.nelz, volfrac=spec.volfrac,
                            rmin=problem.filter_radius or spec.rmin or 1.5, max_iter=self.max_iter,
                            min_iter=min(2, self.max_iter), move=self.move, tol=1.0e-3,
                            checkpoint_dir=self.checkpoint_dir, checkpoint_every=self.checkpoint_every)
        result = run_simp(params, verbose=False, bc_override=lambda a, b, c: (bc.fixed_dofs, bc.free_dofs, F),
                          problem=self.checkpoint_problem, levels=self.levels, device=self.device)
        history = [{"iteration": i + 1, "compliance": float(c)} for i, c in enumerate(result["compliance_history"])]
        summary = {"problem": problem.to_dict(), "backend": "cpu", "linear_solver": "gmg_pcg_fp64_on_b200",
                   "n_iter": int(result["n_iter"]), "final_compliance": float(result["final_compliance"]),
                   "final_grayness": float(result["final_grayness"])}
        return OptimizationResult(problem, result["rho_final"], history, summary)


class SIMPLoop:
    """One SIMP design state on the GPU, advanced by ``step()``.

    A step is one SIMP iteration of the reference path (src/topogpu/solver.py:223-240):
    state solve at the current density, then the OC update; with
    ``use_filter`` the filtered run_simp formulation. ``step_host`` is the same
    step with the density crossing the host boundary (pinned H2D in, D2H out).
    """

    def __init__(self, solver: SIMPSolver, problem: TopologyProblem, *, track_best: bool = False):
        self.solver = solver
        self.problem = problem
        self.state = solver.make_state_solver(problem)
        ctx = self.state.ctx
        dev = self.state.device
        spec = problem.spec
        self.volfrac = float(spec.volfrac)
        self.rho = torch.full((ctx.n_elem,), self.volfrac, dtype=torch.float64, device=dev)
        self.iteration = 0
        self.rmin = None
        self.beta = solver.beta if solver.use_heaviside else None
        self.eta = solver.eta
        self.penal, self.move = float(solver.penal), float(solver.move)
        if solver.use_filter:
            self.rmin = float(problem.filter_radius or spec.rmin or 1.5)
            self.colsum = ctx.filter(self.rmin, torch.ones_like(self.rho), transpose=True)  # H^T 1
        self.rho_phys = self.rho
        # run_simp's best-design bookkeeping (pub_simp_solver.py:477-480,
        # 529-534): the best physical density among iterations with penal >= 3
        # and grayness < 0.25; written into checkpoints
        self.track_best = track_best
        self.min_penal_for_best, self.max_gray_for_best = 3.0, 0.25
        self.compliance_hist: list[float] = []
        self.best_rho = self.rho.clone()
        self.best_compliance, self.best_iteration, self.best_is_valid = float("inf"), 0, False
        self.best_grayness = 4.0 * self.volfrac * (1.0 - self.volfrac)

    def step(self, *, stats: bool = True) -> dict[str, Any]:
        s, ctx = self.solver, self.state.ctx
        if self.beta is not None:
            rho_f = ctx.filter(self.rmin, self.rho)
            rho_phys, dh = ctx.heaviside(rho_f, self.beta, self.eta)
            compliance, dc = self.state.solve(rho_phys, self.penal)
            dc_design = ctx.filter(self.rmin, dc.mul_(dh), transpose=True)
            dv_design = ctx.filter(self.rmin, dh, transpose=True)
            rho_new, _ = ctx.oc_projected(self.rmin, self.rho, dc_design, dv_design, self.beta, self.eta,
                                          self.volfrac, self.move, s.rho_min)
        elif self.rmin is not None:
            rho_phys = ctx.filter(self.rmin, self.rho)
            compliance, dc = self.state.solve(rho_phys, self.penal)
            dc_design = ctx.filter(self.rmin, dc, transpose=True)
            rho_new, _ = ctx.oc_filtered(self.rho, dc_design, self.colsum, self.colsum, self.volfrac, self.move,
                                         s.rho_min)
        else:
            rho_phys = self.rho
            compliance, dc = self.state.solve(self.rho, self.penal)
            rho_new, _ = ctx.oc(self.rho, dc, self.volfrac, self.move, s.rho_min)
        self.rho, self.rho_phys = rho_new, rho_phys
        self.iteration += 1
        compliance = float(compliance)
        if self.track_best:
            self._update_best(compliance)
        row = {"iteration": self.iteration, "compliance": compliance,
               "outer_iters": int(self.state.last_cg_iters), "outer_solver": self.state.last_outer_solver}
        if stats:
            st = ctx.field_stats(self.rho)
            row.update({"rho_mean": st["mean"], "rho_min": st["min"], "rho_max": st["max"],
                        "grayness": st["grayness"]})
        return row

    def _update_best(self, compliance: float) -> None:
        self.compliance_hist.append(compliance)
        gray = self.state.ctx.field_stats(self.rho_phys)["grayness"]
        if compliance < self.best_compliance and self.penal >= self.min_penal_for_best and \
                gray < self.max_gray_for_best:
            self.best_compliance, self.best_rho = compliance, self.rho_phys.clone()
            self.best_iteration, self.best_grayness, self.best_is_valid = self.iteration, gray, True

    def checkpoint_state(self) -> dict[str, Any]:
        """The run_simp checkpoint dictionary (pub_simp_solver.py:597-603)."""
        return {"rho": self.rho.cpu().numpy(), "best_rho": self.best_rho.cpu().numpy(),
                "compliance_hist": np.array(self.compliance_hist, dtype=np.float64),
                "best_compliance": float(self.best_compliance), "best_iteration": int(self.best_iteration),
                "best_is_valid": int(self.best_is_valid), "best_grayness": float(self.best_grayness),
                "penal": self.penal, "rmin": float(self.rmin if self.rmin is not None else self._spec_rmin()),
                "move": self.move, "beta": float(self.beta if self.beta is not None else self.solver.beta),
                "iteration": int(self.iteration)}

    def save_checkpoint(self, path: str) -> None:
        save_checkpoint(path, self.checkpoint_state())

    def restore(self, ck: dict[str, Any]) -> None:
        """Resume from a run_simp checkpoint (pub_simp_solver.py:500-514): the
        design, the best-design record, penal, rmin, move, beta and the
        iteration counter; the next ``step`` is iteration ``ck["iteration"]+1``."""
        dev = self.rho.device
        rho = np.asarray(ck["rho"], dtype=np.float64)
        if rho.shape != (self.rho.numel(),):
            raise ValueError(f"checkpoint rho has {rho.size} entries, expected {self.rho.numel()}")
        self.rho = torch.as_tensor(rho, device=dev).clone()
        self.rho_phys = self.rho
        self.best_rho = torch.as_tensor(np.asarray(ck["best_rho"], dtype=np.float64), device=dev).clone()
        self.best_compliance = float(ck["best_compliance"])
        self.best_iteration = int(ck["best_iteration"])
        self.best_is_valid = bool(int(ck["best_is_valid"]))
        self.best_grayness = float(ck["best_grayness"])
        self.penal, self.move = float(ck["penal"]), float(ck["move"])
        if self.beta is not None:
            self.beta = float(ck["beta"])
        rmin = float(ck["rmin"])
        if self.rmin is not None and abs(rmin - self.rmin) > 1e-6:
            self.rmin = rmin
            self.colsum = self.state.ctx.filter(rmin, torch.ones_like(self.rho), transpose=True)
        self.compliance_hist = [float(c) for c in np.asarray(ck.get("compliance_hist", np.array([])))]
        self.iteration = int(ck["iteration"])

    def _spec_rmin(self) -> float:
        return float(self.problem.filter_radius or self.problem.spec.rmin or 1.5)

    def step_host(self, rho_host: torch.Tensor, out_host: torch.Tensor) -> float:
        """Upload rho (pinned host tensor), run one step, download the new rho."""
        self.rho.copy_(rho_host, non_blocking=True)
        row = self.step(stats=False)
        out_host.copy_(self.rho, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return row["compliance"]

    def close(self):
        self.state.close()


def solve(problem: TopologyProblem, **kwargs: Any) -> OptimizationResult:
    return SIMPSolver(**kwargs).solve(problem)
