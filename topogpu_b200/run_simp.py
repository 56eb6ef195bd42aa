"""``run_simp`` on the GPU: the reference's CPU SIMP driver with its physics on device.

Same call, parameters and result dictionary as the reference's ``run_simp``
(src/gpu_fem/pub_simp_solver.py:88-135 for ``SIMPParams`` / ``StepState``,
412-657 for the driver), for 3-D meshes: filtered and Heaviside-projected
densities, the gated best-design record, the convergence test on the design
change and a compliance window, controller callbacks (``initial_action``,
per-iteration actions with restart and stop, ``finalize_tail``), the tail
phase, and the checkpoint files. Each iteration's physics (filter,
projection, state solve, sensitivity chain and the projected or filtered OC)
runs on the GPU through libtopo_b200; the host keeps the control logic and
reads the scalars it needs, plus the physical density when a callback,
``verbose`` or the checkerboard statistic of ``StepState`` asks for it.

The reference solves the state with SciPy's direct solver (or pyamg above
3,000 DoFs); here it is the FP64 GMG-PCG of ``StateSolver`` to a tight
relative tolerance (``krylov_tol``, default 1e-10), so compliances agree to
about that tolerance rather than bit for bit.
"""

from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from .checkpoint import checkpoint_path, load_checkpoint, save_checkpoint

MIN_ITER_FOR_FALLBACK = 10  # pub_simp_solver.py:488


@dataclass
class SIMPParams:
    """pub_simp_solver.py:88-114 (the AMG fields are accepted and unused)."""

    nelx: int = 60
    nely: int = 30
    nelz: int = 0
    volfrac: float = 0.5
    penal: float = 3.0
    rmin: float = 1.5
    move: float = 0.2
    max_iter: int = 100
    tol: float = 0.01
    compliance_tol: float = 5e-4
    compliance_window: int = 5
    min_iter: int = 50
    tail_default_iters: int = 18
    use_heaviside: bool = True
    beta_init: float = 1.0
    beta_max: float = 32.0
    eta: float = 0.5
    min_penal_for_best: float = 3.0
    max_gray_for_best: float = 0.25
    seed: Optional[int] = None
    checkpoint_dir: Optional[str] = None
    checkpoint_every: int = 10
    amg_ndof_threshold: int = 3000
    amg_rebuild_tol: float = 0.15


@dataclass
class StepState:
    """pub_simp_solver.py:116-135."""

    iteration: int
    compliance: float
    best_compliance: float
    best_iteration: int
    volume_fraction: float
    grayness: float
    best_grayness: float
    checkerboard: float
    obj_slope: float
    rel_change_1: float
    rel_change_5: float
    stagnation_counter: int
    penal: float
    rmin: float
    move: float
    beta: float
    converged: bool
    best_is_valid: bool
    compliance_history: list[float] = field(default_factory=list)


def cantilever_bc_3d(nelx: int, nely: int, nelz: int):
    """run_simp's 3-D "cantilever" preset (pub_simp_solver.py:302-311): the
    x=0 face clamped, a unit load in -y at the centre node of the x=nelx face.
    Returns (fixed, free, F)."""
    nny, nnz = nely + 1, nelz + 1
    ndof = 3 * (nelx + 1) * nny * nnz
    F = np.zeros(ndof)
    tip = nelx * nny * nnz + (nely // 2) * nnz + nelz // 2
    F[3 * tip + 1] = -1.0
    face = np.arange(nny * nnz)
    fixed = np.unique(np.concatenate([3 * face, 3 * face + 1, 3 * face + 2]))
    is_free = np.ones(ndof, dtype=bool)
    is_free[fixed] = False
    return fixed, np.flatnonzero(is_free), F


def grayness(rho: np.ndarray) -> float:
    """pub_simp_solver.py:255."""
    return float(4.0 * np.mean(rho * (1.0 - rho)))


def checkerboard_3d(rho: np.ndarray, nelx: int, nely: int, nelz: int) -> float:
    """Standard deviation of 2x2x2 block means (pub_simp_solver.py:263-270)."""
    R = rho.reshape(nelx, nely, nelz)
    if nelx < 2 or nely < 2 or nelz < 2:
        return 0.0
    b = (R[:-1:2, :-1:2, :-1:2] + R[1::2, :-1:2, :-1:2] + R[:-1:2, 1::2, :-1:2] + R[1::2, 1::2, :-1:2] +
         R[:-1:2, :-1:2, 1::2] + R[1::2, :-1:2, 1::2] + R[:-1:2, 1::2, 1::2] + R[1::2, 1::2, 1::2]) / 8
    return float(np.std(b))


def apply_action(action, penal, rmin, move, beta, rho_new, best_rho, best_is_valid, copy):
    """pub_simp_solver.py:379-386: restart from the best design if one is
    valid, then clip the requested parameters to their ranges."""
    if action.get("restart", False) and best_is_valid:
        rho_new = copy(best_rho)
    if "penal" in action:
        penal = float(np.clip(action["penal"], 1.0, 5.0))
    if "rmin" in action:
        rmin = float(np.clip(action["rmin"], 1.1, 4.0))
    if "move" in action:
        move = float(np.clip(action["move"], 0.03, 0.4))
    if "beta" in action:
        beta = float(np.clip(action["beta"], 1.0, 64.0))
    return penal, rmin, move, beta, rho_new


def tail_defaults(callback, params: SIMPParams) -> dict:
    """pub_simp_solver.py:388-395."""
    tail = {"enabled": False, "tail_iters": params.tail_default_iters, "restart_from_best": True,
            "penal": 4.5, "rmin": 1.2, "move": 0.05, "beta": min(params.beta_max, 32.0)}
    if callback is not None and hasattr(callback, "finalize_tail"):
        custom = callback.finalize_tail(params)
        if custom:
            tail.update(custom)
    return tail


class DeviceFEA:
    """One run_simp iteration's physics on the GPU (``_fea_and_sensitivity``,
    pub_simp_solver.py:342-377): rho_f = H rho, rho_phys = h(rho_f) (or
    rho_f), the state solve at E(rho_phys), dc = H^T(dc_phys h'), dv = H^T h',
    and the OC with the projected (or filtered) volume."""

    def __init__(self, nel, free_mask: np.ndarray, F: np.ndarray, *, krylov_tol=1e-10, max_krylov=2000,
                 levels=4, device=None):
        from .state import StateSolver

        self.nel = tuple(int(v) for v in nel)
        self.st = StateSolver(self.nel, free_mask, F, n_levels=levels, precision="fp64", tol=krylov_tol,
                              maxiter=max_krylov, smoother="chebyshev", device=device)
        self.ctx = self.st.ctx
        self.device = self.st.device
        self.n = self.ctx.n_elem
        self._colsum = {}

    def uniform(self, v: float) -> torch.Tensor:
        return torch.full((self.n,), float(v), dtype=torch.float64, device=self.device)

    def from_host(self, a) -> torch.Tensor:
        return torch.as_tensor(np.asarray(a, dtype=np.float64), device=self.device).clone()

    @staticmethod
    def to_host(x: torch.Tensor) -> np.ndarray:
        return x.detach().cpu().numpy()

    @staticmethod
    def copy(x: torch.Tensor) -> torch.Tensor:
        return x.clone()

    @staticmethod
    def clip(x: torch.Tensor, lo: float, hi: float) -> torch.Tensor:
        return x.clamp(lo, hi)

    def grayness(self, x: torch.Tensor) -> float:
        return float(self.ctx.field_stats(x)["grayness"])

    def _colsum_of(self, rmin: float) -> torch.Tensor:
        if rmin not in self._colsum:
            self._colsum[rmin] = self.ctx.filter(rmin, torch.ones(self.n, dtype=torch.float64, device=self.device),
                                                 transpose=True)
        return self._colsum[rmin]

    def step(self, rho, penal, rmin, move, beta, eta, use_heaviside):
        ctx = self.ctx
        rho_f = ctx.filter(rmin, rho)
        project = use_heaviside and beta > 1e-6
        if project:
            rho_phys, dh = ctx.heaviside(rho_f, beta, eta)
        else:
            rho_phys, dh = rho_f, None
        compliance, dc = self.st.solve(rho_phys, penal)
        if project:
            dc_design = ctx.filter(rmin, dc.mul_(dh), transpose=True)
            dv_design = ctx.filter(rmin, dh, transpose=True)
            rho_new, _ = ctx.oc_projected(rmin, rho, dc_design, dv_design, beta, eta, self._volfrac, move, 1e-3)
        else:
            colsum = self._colsum_of(rmin)
            dc_design = ctx.filter(rmin, dc, transpose=True)
            rho_new, _ = ctx.oc_filtered(rho, dc_design, colsum, colsum, self._volfrac, move, 1e-3)
        change = float((rho_new - rho).abs().max())
        return float(compliance), rho_new, change, rho_phys

    def set_volfrac(self, v: float) -> None:
        self._volfrac = float(v)

    def close(self):
        self.st.close()


def run_simp(params: SIMPParams, callback=None, verbose: bool = False, bc_override=None,
             problem: str = "cantilever", *, krylov_tol: float = 1e-10, levels: int = 4, device=None,
             fea=None) -> dict:
    """The reference's ``run_simp`` (pub_simp_solver.py:412-657) for 3-D
    meshes with the physics on the GPU. ``fea`` replaces the device physics
    with another object of ``DeviceFEA``'s interface."""
    if params.seed is not None:
        np.random.seed(params.seed)
    if params.nelz <= 0:
        raise ValueError("run_simp on the B200 path handles 3-D meshes (nelz > 0) only")
    nelx, nely, nelz = params.nelx, params.nely, params.nelz
    n_elem = nelx * nely * nelz
    if bc_override is not None:
        _, free, F = bc_override(nelx, nely, nelz)
    elif problem == "cantilever":
        _, free, F = cantilever_bc_3d(nelx, nely, nelz)
    else:
        raise ValueError(f"Problem '{problem}' not available for 3D")
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    free_mask = np.zeros(ndof, dtype=np.uint8)
    free_mask[np.asarray(free, dtype=np.int64)] = 1
    own = fea is None
    if own:
        fea = DeviceFEA((nelx, nely, nelz), free_mask, np.asarray(F, dtype=np.float64), krylov_tol=krylov_tol,
                        levels=levels, device=device)
    try:
        return _drive(params, fea, callback, verbose, problem, n_elem)
    finally:
        if own:
            fea.close()


def _drive(params: SIMPParams, fea, callback, verbose, problem, n_elem) -> dict:
    nelx, nely, nelz = params.nelx, params.nely, params.nelz
    fea.set_volfrac(params.volfrac)
    want_host = callback is not None or verbose
    rho = fea.uniform(params.volfrac)
    penal, rmin, move, beta, eta = params.penal, params.rmin, params.move, params.beta_init, params.eta
    if callback is not None and hasattr(callback, "initial_action"):
        init = callback.initial_action(params)
        if init:
            penal, rmin, move, beta, rho = apply_action(init, penal, rmin, move, beta, rho, rho, False, fea.copy)

    best_rho = fea.copy(rho)
    best_compliance, best_iteration, best_is_valid = np.inf, 0, False
    best_grayness = fea.grayness(rho)
    pre_valid_best_compliance, pre_valid_best_iteration = np.inf, 0
    pre_valid_best_grayness = fea.grayness(rho)
    compliance_hist: list[float] = []
    params_log: list[dict] = []
    stagnation_counter = 0
    start_iter = 1

    ckpt_path = None
    if params.checkpoint_dir is not None:
        os.makedirs(params.checkpoint_dir, exist_ok=True)
        ckpt_path = checkpoint_path(params.checkpoint_dir, (nelx, nely, nelz), problem)
        ck = load_checkpoint(ckpt_path)
        if ck is not None:
            rho = fea.from_host(ck["rho"])
            best_rho = fea.from_host(ck["best_rho"])
            best_compliance = float(ck["best_compliance"])
            best_iteration = int(ck["best_iteration"])
            best_is_valid = bool(int(ck["best_is_valid"]))
            pre_valid_best_compliance, pre_valid_best_iteration = best_compliance, best_iteration
            pre_valid_best_grayness = best_grayness
            best_grayness = float(ck["best_grayness"])
            penal, rmin = float(ck["penal"]), float(ck["rmin"])
            move, beta = float(ck["move"]), float(ck["beta"])
            compliance_hist = [float(c) for c in np.asarray(ck.get("compliance_hist", np.array([])))]
            start_iter = int(ck["iteration"]) + 1

    iteration = start_iter - 1
    for iteration in range(start_iter, params.max_iter + 1):
        compliance, rho_new, change, rho_phys = fea.step(rho, penal, rmin, move, beta, eta, params.use_heaviside)
        compliance_hist.append(compliance)
        gray_now = fea.grayness(rho_phys)
        gate_ok = penal >= params.min_penal_for_best and gray_now < params.max_gray_for_best
        if compliance < best_compliance and gate_ok:
            best_compliance, best_rho = compliance, fea.copy(rho_phys)
            best_iteration, best_grayness = iteration, gray_now
            best_is_valid, stagnation_counter = True, 0
        else:
            if (compliance < pre_valid_best_compliance and not best_is_valid and
                    iteration >= MIN_ITER_FOR_FALLBACK):
                # (the reference also keeps this density; it is never returned)
                pre_valid_best_compliance = compliance
                pre_valid_best_iteration, pre_valid_best_grayness = iteration, gray_now
            if compliance >= best_compliance or not gate_ok:
                stagnation_counter += 1

        conv_rho = change < params.tol
        win = compliance_hist[-params.compliance_window:]
        conv_C = (len(win) == params.compliance_window and
                  abs(win[-1] - win[0]) / max(abs(win[0]), 1e-10) < params.compliance_tol)
        conv = conv_rho and conv_C
        slope = (win[-1] - win[0]) / max(len(win) - 1, 1)
        rel1 = 0.0 if len(compliance_hist) < 2 else \
            (compliance_hist[-1] - compliance_hist[-2]) / max(abs(compliance_hist[-2]), 1e-10)
        rel5 = 0.0 if len(compliance_hist) < 6 else \
            (compliance_hist[-1] - compliance_hist[-6]) / max(abs(compliance_hist[-6]), 1e-10)
        rp_host = fea.to_host(rho_phys)
        vf = float(rp_host.sum() / n_elem)
        checker = checkerboard_3d(rp_host, nelx, nely, nelz) if want_host else 0.0
        state = StepState(iteration=iteration, compliance=compliance, best_compliance=best_compliance,
                          best_iteration=best_iteration, volume_fraction=vf, grayness=gray_now,
                          best_grayness=best_grayness, checkerboard=checker, obj_slope=slope,
                          rel_change_1=rel1, rel_change_5=rel5, stagnation_counter=stagnation_counter,
                          penal=penal, rmin=rmin, move=move, beta=beta, converged=conv,
                          best_is_valid=best_is_valid, compliance_history=list(compliance_hist))
        params_log.append({"iter": iteration, "phase": "main", "penal": penal, "rmin": rmin, "move": move,
                           "beta": beta, "compliance": compliance, "best_compliance": best_compliance,
                           "grayness": gray_now, "best_is_valid": best_is_valid, "volume_fraction": vf})
        if verbose:
            print(f"  iter {iteration:3d}  C={compliance:8.4f}  gray={gray_now:.3f}  p={penal:.2f}  "
                  f"beta={beta:.1f}  r={rmin:.2f}  chg={change:.4f}")
        if callback is not None:
            action = callback(state, fea.to_host(rho_new))
            if action:
                penal, rmin, move, beta, rho_new = apply_action(action, penal, rmin, move, beta, rho_new, best_rho,
                                                                best_is_valid, fea.copy)
                if action.get("stop", False) and iteration >= params.min_iter:
                    rho = rho_new
                    break
        rho = rho_new
        if ckpt_path is not None and iteration % params.checkpoint_every == 0:
            save_checkpoint(ckpt_path, dict(
                rho=fea.to_host(rho), best_rho=fea.to_host(best_rho),
                compliance_hist=np.array(compliance_hist), best_compliance=best_compliance,
                best_iteration=best_iteration, best_is_valid=int(best_is_valid), best_grayness=best_grayness,
                penal=penal, rmin=rmin, move=move, beta=beta, iteration=iteration))
        if conv and iteration >= params.min_iter:
            break

    tail = tail_defaults(callback, params)
    tail_iters_run = 0
    if tail.get("enabled", False) and tail.get("tail_iters", 0) > 0:
        if tail.get("restart_from_best", True) and best_is_valid:
            rho = fea.clip(best_rho, 1e-3, 1.0)
        elif tail.get("restart_from_best", True) and not best_is_valid:
            rho = fea.uniform(params.volfrac)
        penal, rmin = float(tail.get("penal", penal)), float(tail.get("rmin", rmin))
        move, beta = float(tail.get("move", move)), float(tail.get("beta", beta))
        for k in range(1, int(tail["tail_iters"]) + 1):
            compliance, rho_new, change, rho_phys = fea.step(rho, penal, rmin, move, beta, eta, params.use_heaviside)
            compliance_hist.append(compliance)
            params_log.append({"iter": iteration + k, "phase": "tail", "penal": penal, "rmin": rmin, "move": move,
                               "beta": beta, "compliance": compliance, "best_compliance": best_compliance,
                               "grayness": fea.grayness(rho_phys), "best_is_valid": best_is_valid,
                               "volume_fraction": float(fea.to_host(rho_phys).sum() / n_elem)})
            rho = rho_new
            tail_iters_run = k

    final_c, _, _, rho_final = fea.step(rho, penal, rmin, move, beta, eta, params.use_heaviside)
    rho_final_h = fea.to_host(rho_final)
    return {
        "compliance_history": compliance_hist,
        "rho_final": rho_final_h,
        "best_rho": fea.to_host(best_rho),
        "best_compliance": best_compliance,
        "best_iteration": best_iteration,
        "final_compliance": final_c,
        "final_grayness": grayness(rho_final_h),
        "best_grayness": best_grayness,
        "best_is_valid": best_is_valid,
        "pre_valid_best_compliance": pre_valid_best_compliance,
        "pre_valid_best_iteration": pre_valid_best_iteration,
        "pre_valid_best_grayness": pre_valid_best_grayness,
        "n_iter": iteration + tail_iters_run,
        "params_log": params_log,
        "tail_config": tail,
        "is_3d": True, "nelx": nelx, "nely": nely, "nelz": nelz,
    }


__all__ = ["SIMPParams", "StepState", "run_simp", "cantilever_bc_3d", "DeviceFEA", "apply_action",
           "tail_defaults", "checkerboard_3d", "grayness"]
