"""GPU parity of the Heaviside projection and the projected-volume OC.

The projection is FP64 tanh arithmetic, so it is compared with the oracle
within a few ulps (rtol 1e-13; its derivative also within a few ulps of beta
in absolute terms, where 1 - tanh^2 cancels). The projected OC takes the same bisection
decisions as the oracle except where a candidate's projected volume lies
within round-off of volfrac, which can only happen once the lambda bracket is
already tiny; the number of evaluations is fixed by the bracket (1e9 halved
down to 1e-9), so it must match exactly, and the candidates agree to the
bracket's slack (rtol 1e-8).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import design, fem

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _t(x):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=DEV)


def _ctx(nel):
    from topogpu_b200.context import TopoContext

    bc = fem.cantilever_bc(nel)
    ctx = TopoContext(nel, n_levels=1, mode="fp64", smoother="reference")
    mask = np.zeros(bc.ndof, dtype=np.uint8)
    mask[bc.free] = 1
    ctx.set_problem(torch.as_tensor(mask, device=DEV), torch.as_tensor(bc.F, device=DEV))
    return ctx


@pytest.mark.parametrize("beta", [0.0, 1.0, 8.0, 32.0, 64.0])
def test_heaviside_matches_oracle(cuda_dev, beta):
    nel = (12, 6, 5)
    ctx = _ctx(nel)
    x = np.random.default_rng(2).uniform(0.0, 1.0, ctx.n_elem)
    x[:3] = (0.0, 0.5, 1.0)
    phys, dh = ctx.heaviside(_t(x), beta, 0.5)
    np.testing.assert_allclose(phys.cpu().numpy(), design.heaviside(x, beta, 0.5), rtol=1e-13, atol=1e-15)
    # h' = beta (1 - t^2) / den cancels where tanh saturates (|t| -> 1): one ulp
    # of t there is an absolute error of about beta * 2e-16 in h'
    np.testing.assert_allclose(dh.cpu().numpy(), design.heaviside_deriv(x, beta, 0.5), rtol=1e-13,
                               atol=4e-15 * max(beta, 1.0))
    only = ctx.heaviside(_t(x), beta, 0.5, want_deriv=False)
    assert torch.equal(only, phys)


@pytest.mark.parametrize("nel,rmin,beta,eta", [((24, 12, 6), 1.5, 1.0, 0.5), ((24, 12, 6), 1.5, 8.0, 0.5),
                                               ((7, 5, 3), 2.0, 32.0, 0.4), ((10, 6, 4), 1.5, 0.0, 0.5)])
def test_oc_projected_matches_oracle(cuda_dev, nel, rmin, beta, eta):
    H = design.filter_matrix(nel, rmin)
    n = H.shape[0]
    rng = np.random.default_rng(5)
    rho = rng.uniform(0.01, 0.6, n)  # volfrac 0.3 reachable within the move limits
    rf = H @ rho
    dh = design.heaviside_deriv(rf, beta, eta)
    dc = H.T @ (-rng.gamma(1.0, 1.0, n) * dh)
    dv = H.T @ dh
    ref, kref = design.oc_update_projected(rho, dc, dv, 0.3, 0.2, H, beta, eta)
    ctx = _ctx(nel)
    out, k = ctx.oc_projected(rmin, _t(rho), _t(dc), _t(dv), beta, eta, 0.3, 0.2)
    assert k == kref
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-8, atol=1e-12)
    # the projected volume of the result sits at volfrac to the bracket's slack
    vol = design.heaviside(H @ out.cpu().numpy(), beta, eta).mean()
    assert abs(vol - 0.3) < 1e-6


def test_oc_projected_rejects_aliasing(cuda_dev):
    ctx = _ctx((6, 4, 3))
    x = torch.full((ctx.n_elem,), 0.3, dtype=torch.float64, device=DEV)
    with pytest.raises(RuntimeError, match="alias"):
        ctx.oc_projected(1.5, x, -torch.ones_like(x), torch.ones_like(x), 1.0, out=x)


@pytest.mark.parametrize("beta", [1, 8])
def test_simp_heaviside_matches_run_simp(cuda_dev, beta):
    """Three SIMP iterations with projection through the public driver
    against the reference run_simp (use_heaviside, beta fixed)."""
    import topogpu_b200 as tg

    g = load_golden("run_simp_heaviside")
    p = tg.gallery.benchmark_cantilever((24, 12, 6), volfrac=0.3, filter_radius=1.5)
    res = tg.SIMPSolver(backend="cuda", tol=1e-10, max_krylov=800, max_iter=3, move=0.2, precision="fp64",
                        use_filter=True, use_heaviside=True, beta=float(beta)).solve(p)
    comp = [r["compliance"] for r in res.history]
    np.testing.assert_allclose(comp, g[f"compliance_b{beta}"], rtol=1e-8)


def test_simp_heaviside_loop_matches_oracle_with_beta_change(cuda_dev):
    """SIMPLoop with beta raised between steps (the way run_simp's
    continuation changes it) against the oracle's fixed-beta loop run in two
    legs."""
    import topogpu_b200 as tg
    from topogpu_b200.solver import SIMPLoop

    nel = (24, 12, 6)
    p = tg.gallery.benchmark_cantilever(nel, volfrac=0.3, filter_radius=1.5)
    s = tg.SIMPSolver(backend="cuda", tol=1e-11, max_krylov=800, move=0.2, precision="fp64", use_filter=True,
                      use_heaviside=True, beta=1.0)
    loop = SIMPLoop(s, p)
    try:
        comp = [loop.step(stats=False)["compliance"] for _ in range(2)]
        loop.beta = 4.0
        comp += [loop.step(stats=False)["compliance"] for _ in range(2)]
        rho_gpu = loop.rho.cpu().numpy()
    finally:
        loop.close()
    bc = fem.cantilever_bc(nel)
    H = design.filter_matrix(nel, 1.5)
    rho = np.full(H.shape[0], 0.3)
    ref = []
    for beta in (1.0, 1.0, 4.0, 4.0):
        rf = H @ rho
        rp = design.heaviside(rf, beta, 0.5)
        U = fem.direct_solve(1e-9 + (1 - 1e-9) * rp**3, nel, bc)
        ref.append(float(bc.F @ U))
        dcp = -3.0 * (1 - 1e-9) * rp**2 * fem.element_energy(U, nel)
        dh = design.heaviside_deriv(rf, beta, 0.5)
        rho, _ = design.oc_update_projected(rho, H.T @ (dcp * dh), H.T @ dh, 0.3, 0.2, H, beta, 0.5)
    np.testing.assert_allclose(comp, ref, rtol=1e-8)
    np.testing.assert_allclose(rho_gpu, rho, rtol=1e-6, atol=1e-8)


def test_resume_from_reference_checkpoint(cuda_dev, tmp_path):
    """Resume the filtered SIMP loop from the checkpoint run_simp wrote after
    iteration 2 of config 0: iteration 3 gives run_simp's third compliance,
    and the checkpoint written after it carries the whole history."""
    import shutil

    import topogpu_b200 as tg
    from conftest import GOLDEN
    from topogpu_b200.checkpoint import load_checkpoint

    for ext in (".npz", ".json"):
        shutil.copy(GOLDEN / f"ckpt_24x12x6_cantilever{ext}", tmp_path / f"ckpt_24x12x6_cantilever{ext}")
    g = load_golden("run_simp")
    p = tg.gallery.benchmark_cantilever((24, 12, 6), volfrac=0.3, filter_radius=1.5)
    res = tg.SIMPSolver(backend="cuda", tol=1e-10, max_krylov=800, max_iter=3, move=0.2, precision="fp64",
                        use_filter=True, checkpoint_dir=str(tmp_path), checkpoint_every=1).solve(p)
    assert [r["iteration"] for r in res.history] == [3]
    np.testing.assert_allclose(res.history[0]["compliance"], g["compliance"][2], rtol=1e-8)
    ck = load_checkpoint(str(tmp_path / "ckpt_24x12x6_cantilever"))
    assert ck["iteration"] == 3
    np.testing.assert_allclose(ck["compliance_hist"], g["compliance"], rtol=1e-8)


def test_interrupted_run_resumes_to_same_history(cuda_dev, tmp_path):
    """Two iterations, a checkpoint, then a fresh solver resuming to four
    iterations gives the compliances of one uninterrupted four-iteration run."""
    import topogpu_b200 as tg

    p = tg.gallery.benchmark_cantilever((24, 12, 6), volfrac=0.3, filter_radius=1.5)
    kw = dict(backend="cuda", tol=1e-10, max_krylov=800, move=0.2, precision="fp64", use_filter=True,
              use_heaviside=True, beta=2.0)
    full = [r["compliance"] for r in tg.SIMPSolver(max_iter=4, **kw).solve(p).history]
    tg.SIMPSolver(max_iter=2, checkpoint_dir=str(tmp_path), checkpoint_every=2, **kw).solve(p)
    rest = tg.SIMPSolver(max_iter=4, checkpoint_dir=str(tmp_path), checkpoint_every=2, **kw).solve(p)
    assert [r["iteration"] for r in rest.history] == [3, 4]
    np.testing.assert_allclose([r["compliance"] for r in rest.history], full[2:], rtol=1e-7)
