"""Differentiable compliance on the 48x24x24 cantilever (rho ~ U[0.05, 1],
density filter rmin 1.5): autograd gradients against central finite
differences, FP32 against FP64, the adjoint of a non-self-adjoint objective,
and a short torch-optimizer run under the volume constraint.

The finite differences difference the discrete compliance C(rho) = F^T K(rho)^-1 F,
each value evaluated in the energy form 2 F.u - u.K u (error quadratic in the
PCG residual) after FP64 GMG-PCG solves to relres 1e-14.
"""

import numpy as np
import pytest
import torch

from topogpu_b200.autograd import compliance, density_filter, energy_compliance, linear_objective
from topogpu_b200.bc import cantilever_edge_load
from topogpu_b200.state import StateSolver

NEL3 = (48, 24, 24)
NE3 = 48 * 24 * 24
RMIN = 1.5


def _state(precision, tol, levels=4):
    mask, F = cantilever_edge_load(NEL3)
    return StateSolver(NEL3, mask, F, n_levels=levels, precision=precision, tol=tol, maxiter=4000, device="cuda")


def _rho(seed=3):
    g = torch.Generator().manual_seed(seed)
    return (0.05 + 0.95 * torch.rand(NE3, generator=g, dtype=torch.float64)).cuda()


def _grad(state, rho0):
    rho = rho0.clone().requires_grad_(True)
    c = compliance(density_filter(rho, state.ctx, RMIN), state)
    c.backward()
    return float(c.detach()), rho.grad.detach().clone()


@pytest.mark.gpu
def test_compliance_gradient_matches_central_fd_fp64(cuda_dev):
    st = _state("fp64", 1e-14)
    rho0 = _rho()
    c, g_ad = _grad(st, rho0)
    assert st.last_converged
    # the energy form and F.u agree at this tolerance
    e = energy_compliance(st.ctx.filter(RMIN, rho0), st)
    assert abs(e - c) <= 1e-11 * abs(c)
    idx = np.random.default_rng(7).choice(NE3, 64, replace=False)
    h = 1e-6
    fd = []
    for i in idx.tolist():
        rp, rm = rho0.clone(), rho0.clone()
        rp[i] += h
        rm[i] -= h
        jp = energy_compliance(st.ctx.filter(RMIN, rp), st)
        jm = energy_compliance(st.ctx.filter(RMIN, rm), st)
        fd.append((jp - jm) / (2 * h))
    fd = torch.tensor(fd, dtype=torch.float64)
    ad = g_ad[torch.from_numpy(idx).cuda()].cpu()
    rel = float((ad - fd).norm() / fd.norm())
    print(f"autograd vs central FD (h=1e-6, 64 elements): rel L2 {rel:.3e}")
    assert rel < 1e-5
    st.close()


@pytest.mark.gpu
def test_compliance_gradient_fp32_close_to_fp64(cuda_dev):
    rho0 = _rho()
    s64 = _state("fp64", 1e-12)
    c64, g64 = _grad(s64, rho0)
    s32 = _state("fp32", 1e-7)
    c32, g32 = _grad(s32, rho0)
    assert abs(c32 - c64) <= 1e-5 * abs(c64)
    rel = float((g32 - g64).norm() / g64.norm())
    assert rel < 1e-4, rel
    s64.close()
    s32.close()


@pytest.mark.gpu
def test_linear_objective_adjoint_matches_fd(cuda_dev):
    st = _state("fp64", 1e-14)
    rho0 = _rho(5)
    # J = L.u with L a seeded combination of loads on the free DoFs (not F)
    gen = torch.Generator().manual_seed(11)
    L = (torch.randn(st.ctx.ndof, generator=gen, dtype=torch.float64)).cuda() * st.free_mask
    rho = rho0.clone().requires_grad_(True)
    J = linear_objective(rho, st, L)
    J.backward()
    g_ad = rho.grad.detach().clone()
    idx = np.random.default_rng(13).choice(NE3, 16, replace=False)
    h = 1e-5
    fd = []
    with torch.no_grad():
        for i in idx.tolist():
            vals = []
            for sgn in (1.0, -1.0):
                r = rho0.clone()
                r[i] += sgn * h
                st.solve(r)
                vals.append(float(torch.dot(L, st.displacement())))
            fd.append((vals[0] - vals[1]) / (2 * h))
    fd = torch.tensor(fd, dtype=torch.float64)
    rel = float((g_ad[torch.from_numpy(idx).cuda()].cpu() - fd).norm() / fd.norm())
    print(f"adjoint vs central FD (h=1e-5, 16 elements): rel L2 {rel:.3e}")
    assert rel < 1e-4
    # with L = F the adjoint gradient is the compliance gradient
    rho = rho0.clone().requires_grad_(True)
    linear_objective(rho, st, st.F).backward()
    ga = rho.grad.detach().clone()
    rho2 = rho0.clone().requires_grad_(True)
    compliance(rho2, st).backward()
    assert float((ga - rho2.grad).norm() / rho2.grad.norm()) < 1e-9
    st.close()


def _volume_projection(theta, volfrac, rho_min=1e-3):
    """rho = rho_min + (1 - rho_min) sigmoid(theta + s), s by bisection so that mean(rho) = volfrac."""
    lo, hi = -60.0, 60.0
    with torch.no_grad():
        for _ in range(100):
            s = 0.5 * (lo + hi)
            m = float((rho_min + (1 - rho_min) * torch.sigmoid(theta + s)).mean())
            lo, hi = (s, hi) if m < volfrac else (lo, s)
    return rho_min + (1 - rho_min) * torch.sigmoid(theta + 0.5 * (lo + hi))


@pytest.mark.gpu
def test_torch_optimizer_steps_under_volume_constraint(cuda_dev):
    st = _state("mixed", 1e-6)
    theta = torch.zeros(NE3, dtype=torch.float64, device="cuda", requires_grad=True)
    opt = torch.optim.Adam([theta], lr=0.2)
    hist = []
    for _ in range(20):
        rho = _volume_projection(theta, 0.3)
        c = compliance(density_filter(rho, st.ctx, RMIN), st)
        opt.zero_grad()
        c.backward()
        with torch.no_grad():
            # the volume projection absorbs uniform moves: step in the
            # mean-free part of the gradient
            theta.grad -= theta.grad.mean()
        opt.step()
        hist.append(float(c.detach()))
        assert abs(float(rho.mean()) - 0.3) < 1e-6
    print("compliance over 20 Adam steps:", [round(v, 4) for v in hist])
    assert hist[-1] < 0.8 * hist[0]
    st.close()
