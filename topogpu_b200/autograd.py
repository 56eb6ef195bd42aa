"""Differentiable state solve: compliance and linear objectives as torch autograd functions.

``compliance(rho, state)`` runs the GMG-PCG state solve of ``StateSolver``
in its forward pass and, in its backward pass, scales the upstream gradient
by the element-energy sensitivity computed on the device by the CUDA kernel
of ``topo_sensitivity`` (compliance is self-adjoint, so no second solve:
dc/drho_e = -p rho_e^(p-1) (E0-Emin) u_e^T KE u_e, the formula of
SolverV4.solve, src/gpu_fem/solver_v4.py:244-251).

``density_filter(x, ctx, rmin)`` is the stencil density filter as an
autograd function (forward H x, backward H^T g, both on the device), so a
filtered compliance chains through H^T as run_simp does by hand
(src/gpu_fem/pub_simp_solver.py:347-371).

``linear_objective(rho, state, L)`` differentiates J = L^T u, which is not
self-adjoint: its backward pass solves the adjoint system K lam = L with the
same GMG hierarchy and contracts lam_e^T KE u_e (``topo_sensitivity_adjoint``).

``energy_compliance(rho, state)`` evaluates the same discrete compliance in
the energy form 2 F.u - u.K u, whose error is quadratic in the solve error;
finite-difference checks use it.
"""

from __future__ import annotations

import torch

from .state import StateSolver


class _Compliance(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho, state: StateSolver, penal: float):
        c, dc = state.solve(rho.detach(), penal)
        ctx.save_for_backward(dc)
        return torch.tensor(c, dtype=torch.float64, device=rho.device)

    @staticmethod
    def backward(ctx, g):
        (dc,) = ctx.saved_tensors
        return g * dc, None, None


def compliance(rho: torch.Tensor, state: StateSolver, penal: float = 3.0) -> torch.Tensor:
    """Compliance F.u(rho) with a device-side adjoint gradient (float64 scalar)."""
    return _Compliance.apply(rho, state, float(penal))


class _Filter(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, tctx, rmin: float):
        ctx.tctx, ctx.rmin = tctx, rmin
        return tctx.filter(rmin, x.detach().contiguous(), transpose=False)

    @staticmethod
    def backward(ctx, g):
        return ctx.tctx.filter(ctx.rmin, g.contiguous(), transpose=True), None, None


def density_filter(x: torch.Tensor, tctx, rmin: float) -> torch.Tensor:
    """H x with the linear-hat filter of radius rmin; gradient H^T g."""
    return _Filter.apply(x, tctx, float(rmin))


class _Linear(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho, state: StateSolver, L, penal: float, tol: float, maxiter: int):
        rho = rho.detach()
        state.solve(rho, penal)
        u = state.displacement().clone()
        b = (L.to(torch.float64) * state.free_mask).contiguous()
        lam = torch.zeros_like(u)
        it, rr, ok = state.ctx.pcg(b, lam, tol, maxiter)
        if not ok:
            raise RuntimeError(f"adjoint solve did not converge ({it} iterations, relres {rr:.3e})")
        dj = state.ctx.sensitivity_adjoint(u, lam, rho, penal, state.E0, state.Emin)
        ctx.save_for_backward(dj)
        return torch.dot(b, u)

    @staticmethod
    def backward(ctx, g):
        (dj,) = ctx.saved_tensors
        return g * dj, None, None, None, None, None


def linear_objective(rho: torch.Tensor, state: StateSolver, L: torch.Tensor, penal: float = 3.0,
                     tol: float | None = None, maxiter: int | None = None) -> torch.Tensor:
    """J = L^T u(rho) (fixed DoFs of L ignored); backward uses one adjoint solve."""
    return _Linear.apply(rho, state, L, float(penal), state.tol if tol is None else float(tol),
                         state.maxiter if maxiter is None else int(maxiter))


@torch.no_grad()
def energy_compliance(rho: torch.Tensor, state: StateSolver, penal: float = 3.0) -> float:
    """2 F.u - u.K(rho) u after a state solve: the discrete compliance with an
    error quadratic in the solve error. u.K u is summed as sum_e E_e u_e^T KE u_e
    (element energies from the sensitivity kernel, all non-negative), so the
    sum has no cancellation."""
    state.solve(rho, penal)
    u = state.displacement()
    rho = rho.contiguous()
    E = state.ctx.modulus(rho, penal, state.E0, state.Emin)
    # with penal 1 the kernel returns -(E0-Emin) u_e^T KE u_e
    ce = state.ctx.sensitivity(u, rho, 1.0, state.E0, state.Emin) / -(state.E0 - state.Emin)
    return float(2.0 * torch.dot(state.F * state.free_mask, u) - torch.dot(E, ce))
