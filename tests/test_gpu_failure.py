"""Failure detection without a GPU fault.

* Bounded waits: the test hook topo_debug_tc_wait makes the tensor-core
  K.u's converter warps withhold their first arrival, so the MMA role's
  mbarrier wait runs out (after a short poll limit). The kernel raises its
  per-device error flag, drains its copies, frees its tensor memory and
  exits; the entry point returns an error, and the same context then
  computes the right result. No trap, no fault, no endless loop.
* Non-finite inputs injected on the host: NaN moduli make topo_gmg_setup
  fail, an Inf right-hand side or a NaN initial guess makes topo_pcg fail,
  each with a message; the context stays usable. The reference's nearest
  behaviour is its PCG retry from a cold start when a warm-started solve
  does not converge (src/gpu_fem/solver_v4.py:201-209).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import fem

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _ctx(nel, mode="mixed", n_levels=1):
    from topogpu_b200.context import TopoContext

    bc = fem.cantilever_bc(nel)
    mask = np.zeros(bc.ndof, dtype=np.uint8)
    mask[bc.free] = 1
    ctx = TopoContext(nel, n_levels=n_levels, mode=mode, fine_degree=3)
    ctx.set_problem(torch.tensor(mask, device=DEV), torch.tensor(bc.F, device=DEV))
    return ctx, bc, mask


def test_tensor_core_wait_timeout_returns_error(cuda_dev):
    from topogpu_b200 import _lib

    lib = _lib.load()
    nel = (24, 12, 6)
    ctx, bc, mask = _ctx(nel)
    rng = np.random.default_rng(0)
    E = fem.simp_modulus(rng.uniform(0.01, 1.0, int(np.prod(nel)))).astype(np.float32)
    u = (rng.standard_normal(bc.ndof) * mask).astype(np.float32)
    Et = torch.tensor(E, device=DEV)
    ub = torch.tensor(u, device=DEV).to(torch.bfloat16)
    assert lib.topo_debug_tc_wait(1, 1 << 14) == 0
    try:
        ctx.level0_apply(ub, Et, "store")  # asynchronous: returns before the wait runs out
        with pytest.raises(RuntimeError, match="timed out"):
            ctx.wait_status()
        ctx.level0_apply(ub, Et, "store")
        torch.cuda.synchronize()
    finally:
        lib.topo_debug_tc_wait(0, 0)
    # a later asynchronous call reports the earlier launch's timeout before launching
    with pytest.raises(RuntimeError, match="earlier launch timed out"):
        ctx.level0_apply(ub, Et, "store")
    # the context and the device are still usable, and the error flag was cleared
    y = ctx.level0_apply(ub, Et, "store").cpu().numpy()
    ref = fem.matvec_full(fem.bf16_round(u), E, nel, "bf16").astype(np.float64)
    ref[mask == 0] = 0.0
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-5
    ctx.close()


def test_nan_moduli_fail_setup(cuda_dev):
    nel = (16, 8, 8)
    ctx, bc, _ = _ctx(nel, mode="fp64", n_levels=3)
    E = fem.simp_modulus(np.full(int(np.prod(nel)), 0.3))
    bad = E.copy()
    bad[17] = np.nan
    with pytest.raises(RuntimeError, match="NaN or Inf"):
        ctx.gmg_setup(torch.tensor(bad, device=DEV))
    rho = np.full(int(np.prod(nel)), 0.3)
    rho[5] = np.inf
    with pytest.raises(RuntimeError, match="NaN or Inf"):
        ctx.gmg_setup(ctx.modulus(torch.tensor(rho, device=DEV)))
    # a valid setup afterwards solves normally
    ctx.gmg_setup(torch.tensor(E, device=DEV))
    x = torch.zeros(bc.ndof, dtype=torch.float64, device=DEV)
    it, rr, ok = ctx.pcg(torch.tensor(bc.F, device=DEV), x, tol=1e-8, maxiter=300)
    assert ok and rr < 1e-8
    ctx.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_nonfinite_rhs_or_guess_fail_pcg(cuda_dev, mode):
    nel = (16, 8, 8)
    ctx, bc, _ = _ctx(nel, mode=mode, n_levels=3)
    E = fem.simp_modulus(np.full(int(np.prod(nel)), 0.3))
    ctx.gmg_setup(torch.tensor(E, device=DEV))
    F = bc.F.copy()
    F[bc.free[3]] = np.inf
    x = torch.zeros(bc.ndof, dtype=torch.float64, device=DEV)
    with pytest.raises(RuntimeError, match="right-hand side"):
        ctx.pcg(torch.tensor(F, device=DEV), x, tol=1e-6, maxiter=100)
    x0 = torch.zeros(bc.ndof, dtype=torch.float64, device=DEV)
    x0[bc.free[7]] = float("nan")
    with pytest.raises(RuntimeError, match="initial guess"):
        ctx.pcg(torch.tensor(bc.F, device=DEV), x0, tol=1e-6, maxiter=100)
    x = torch.zeros(bc.ndof, dtype=torch.float64, device=DEV)
    it, rr, ok = ctx.pcg(torch.tensor(bc.F, device=DEV), x, tol=1e-6, maxiter=300)
    assert ok and rr < 1e-6
    ctx.close()
